"""CPU check that the Mosscap-side hook adapter (include/mosscap_b200_hooks.hpp)
compiles against the reference's own Simulation type, i.e. that it is the
binding a Mosscap maintainer can add. Needs the reference sources; no GPU."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from oracle.oracle import REF_SOURCE as REF


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference sources not present")
def test_adapter_compiles_against_reference_simulation():
    src = """
#include "Simulation.hpp"
#include "mosscap_b200_hooks.hpp"
void install_into(Mosscap::Simulation& sim) {
    auto ctx = mosscap_b200::install(sim);
    (void)ctx;
}
"""
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "t.cpp")
        open(f, "w").write(src)
        r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-w", f"-I{REF}",
                            "-I" + os.path.join(ROOT, "oracle", "ref_shim", "include"),
                            "-I" + os.path.join(ROOT, "include"),
                            "-I" + os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include"), f],
                           capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def _adapter_case(name):
    """(problem, steps, gravity, user_bc) of an adapter run."""
    import numpy as np
    from mosscap_b200 import problems as P
    if name == "kh2d_64":
        return P.kelvin_helmholtz_2d(64, seed=0), 20, None, False
    if name == "sedov3d_12":
        return P.sedov_3d(12).with_scheme(output_delta=0.004), 10, None, False
    # a 2D box whose x-start face is a user boundary (an inflow that reads
    # sim.dt_sub), periodic in y, zero-gradient at x-end
    stepper = "rk2" if name == "user_bc_rk2_gravity" else "ssprk4"
    q = P.random_state(2, 48, 40, 1, ng=3, seed=21)
    p = P.Problem("user_bc", 2, 48, 40, ng=3, dx=1.0 / 48,
                  bc=("userfn", "zerograd", "periodic", "periodic", "zerograd", "zerograd"),
                  reconstruction="muscl", slope_limiter="minmod", riemann_solver="hllc", time_stepper=stepper,
                  gamma=1.4, max_cfl=0.4, max_time=1.0, output_delta=0.01, Q=np.ascontiguousarray(q))
    grav = (0.0, -0.5, 0.0) if name == "user_bc_rk2_gravity" else None
    return p, 12, grav, True


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["kh2d_64", "sedov3d_12", "user_bc_rk2_gravity", "user_bc_ssprk4"])
def test_adapter_drives_reference_simulation(gpu_lib, case, tmp_path):
    """The reference's own Simulation, run by the reference's main loop, with
    the hooks mosscap_b200::install() puts in place: the state, the W array,
    the dt sequence and the clock must equal the reference's own hooks' bit
    for bit (source/main.cpp:54-72, Boundaries.hpp:146-148, Output.cpp:226-229)."""
    import ctypes
    import json
    import numpy as np
    from oracle import oracle as O
    if not os.path.exists(O.ADAPTER_CHECK):
        pytest.skip("adapter check not built (it needs the reference sources at build time)")
    p, steps, grav, user_bc = _adapter_case(case)
    cfg = O.OracleConfig(**p.scheme_fields()).to_c()
    (tmp_path / "config.bin").write_bytes(ctypes.string_at(ctypes.addressof(cfg), ctypes.sizeof(cfg)))
    (tmp_path / "q0.bin").write_bytes(np.ascontiguousarray(p.Q, dtype=np.float64).tobytes())
    if grav is not None:
        (tmp_path / "gravity.bin").write_bytes(np.asarray(grav, dtype=np.float64).tobytes())
    cmd = [O.ADAPTER_CHECK, str(tmp_path), str(steps)] + (["user_bc"] if user_bc else [])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    clocks = json.loads(r.stdout.strip().splitlines()[-1])
    assert clocks["ref"] == clocks["lib"], clocks
    assert clocks["lib"]["steps"] == steps

    def load(name):
        return np.fromfile(str(tmp_path / name), dtype=np.float64).view(np.uint64)

    for part in ("dt", "q", "w"):
        a, b = load(f"ref_{part}.bin"), load(f"lib_{part}.bin")
        assert a.size == b.size and a.size > 0, part
        ndiff = int(np.count_nonzero(a != b))
        assert ndiff == 0, f"{case}: {ndiff} of {a.size} values of {part} differ"
