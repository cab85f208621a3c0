"""GPU parity: the sm_100a kernels (through the C ABI) against the reference.

FP64 results must be bit-identical: states compared as bit patterns, dt
sequences bit for bit. Reference values come from the committed golden
fixtures (generated by the reference's own code, tests/golden/make_golden.py)
and, at sizes beyond the fixtures, from the C restatement of the reference
(oracle/liboracle_port.so, itself pinned bit-exact to the reference)."""
import hashlib
import json
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from mosscap_b200 import problems as P

pytestmark = pytest.mark.gpu


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


def _sim(p, precision="fp64"):
    from mosscap_b200.hydro import HydroSim
    return HydroSim(p, precision=precision)


def _oracle(O, p):
    s = O.OracleSim(O.OracleConfig(**p.scheme_fields()), "port")
    if p.gravity is not None:
        s.set_gravity(p.gravity)
    s.set_Q(p.Q)
    s.fill_bcs()
    return s


def _assert_same(a, b, what=""):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        raise AssertionError(f"{what}: shape {a.shape} vs {b.shape}: {a.ravel()[:8]} vs {b.ravel()[:8]}")
    if not np.array_equal(_bits(a), _bits(b)):
        d = np.abs(np.asarray(a) - np.asarray(b))
        idx = np.argwhere(_bits(a) != _bits(b))
        raise AssertionError(f"{what}: {len(idx)} values differ, max |diff| {np.nanmax(d):.3e}, first {idx[:4]}")


@pytest.mark.parametrize("name", ["sod_1d", "kh_2d_64", "sedov_3d_12"])
@pytest.mark.parametrize("loop", ["host", "device"])
def test_headline_fixtures(gpu_lib, name, loop):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    p = {"sod_1d": P.sod_1d(1024), "kh_2d_64": P.kelvin_helmholtz_2d(64, seed=0),
         "sedov_3d_12": P.sedov_3d(12).with_scheme(output_delta=0.004)}[name]
    sim = _sim(p)
    sim.fill_bcs()
    _assert_same(sim.get_Q(), g["q0"], "fill_bcs")
    dts = sim.run(len(g["dts"]), device_loop=(loop == "device"))
    _assert_same(dts, g["dts"], "dt sequence")
    _assert_same(sim.get_Q(), g["q1"], "final state")
    assert sim.time == float(g["time"])
    assert sim.status() == 0
    assert sim.launch_count() > 0


def test_scheme_sweep_against_reference(gpu_lib):
    """216 cases: every reconstruction x limiter x solver x stepper in 1D, 2D
    and 3D with mixed boundary kinds (wall, periodic, symmetric, diode,
    zero-gradient) and a passive tracer, plus the gravity source term with
    every stepper in 1D / 2D / 3D, against the reference's hashes."""
    gold = json.load(open(os.path.join(GOLDEN, "sweep.json")))
    from make_golden import sweep_cases
    bad = []
    for name, p, steps, seed in sweep_cases():
        gcase = gold[name]
        sim = _sim(p)
        sim.fill_bcs()
        if _sha(sim.get_Q()) != gcase["q0_sha256"]:
            bad.append((name, "fill_bcs"))
            continue
        dts = sim.run(steps, device_loop=(seed % 2 == 0))
        if [int(x) for x in _bits(dts)] != gcase["dt_bits"]:
            bad.append((name, "dt"))
        elif _sha(sim.get_Q()) != gcase["q1_sha256"]:
            bad.append((name, "state"))
        sim.close()
    assert not bad, bad


@pytest.mark.parametrize("ndim,n", [(1, 700), (2, 97), (3, 35)])
def test_fill_bcs_and_compute_dt_all_kinds(gpu_lib, oracle_port, ndim, n):
    """Every built-in boundary kind including constant faces and corners,
    on tile-unaligned sizes; then compute_dt (min over every cell) bit-exact."""
    O = oracle_port
    bcc = np.zeros((6, 5))
    nh = 2 + ndim
    for f in range(6):
        bcc[f, 0] = 0.5 + 0.25 * f
        bcc[f, 1:nh - 1] = 0.1 * (f - 2)
        bcc[f, nh - 1] = 2.0 + f
    kinds = {1: ("constant", "symmetricoutflowdiode", "", "", "", ""),
             2: ("wall", "constant", "symmetricoutflowdiode", "zerograd", "", ""),
             3: ("symmetric", "constant", "periodic", "periodic", "symmetricoutflowdiode", "wall")}[ndim]
    bc = tuple(k or "zerograd" for k in kinds)
    q = P.random_state(ndim, n, n, n, ng=3, seed=11 + ndim)
    p = P.Problem("bcs", ndim, n, n if ndim > 1 else 1, n if ndim > 2 else 1, ng=3, dx=1.0 / n, bc=bc,
                  bc_const=bcc, reconstruction="weno5z", riemann_solver="hllc", time_stepper="ssprk3",
                  max_cfl=0.7, max_time=0.3, output_delta=0.07, Q=q)
    o = _oracle(O, p)
    sim = _sim(p)
    sim.fill_bcs()
    _assert_same(sim.get_Q(), o.get_Q(), "fill_bcs")
    assert sim.compute_dt() == o.compute_dt()
    assert sim.compute_dt(clamp=False) == o.cfl_min() * p.max_cfl
    # three steps through the host-driven hooks
    for _ in range(3):
        dt = o.compute_dt()
        assert sim.compute_dt() == dt
        o.time_step(dt)
        sim.time_step(dt)
    _assert_same(sim.get_Q(), o.get_Q(), "state after 3 steps")


def test_kh_256_against_port(gpu_lib, oracle_port):
    """Headline scheme (WENO5-Z + HLLC + SSPRK3, periodic) on a grid with
    partial tiles in both directions: 10 steps bit-exact."""
    p = P.kelvin_helmholtz_2d(256, seed=3)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(10)
    sim = _sim(p)
    sim.fill_bcs()
    dts = sim.run(10)
    _assert_same(dts, ref_dts, "dt")
    _assert_same(sim.get_Q(), o.get_Q(), "state")


def test_sedov_32_to_t005_against_port(gpu_lib, oracle_port):
    """3D Sedov (PPM/MC + HLL, SSPRK3, zero-gradient) to t = 0.05 at 32^3."""
    p = P.sedov_3d(32)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(10 ** 6)
    sim = _sim(p)
    sim.fill_bcs()
    dts = sim.run(10 ** 6)
    assert sim.time == o.time == 0.05
    _assert_same(dts, ref_dts, "dt")
    _assert_same(sim.get_Q(), o.get_Q(), "state")


def test_status_flags_and_errors(gpu_lib):
    from mosscap_b200 import capi
    p = P.sod_1d(256)
    q = p.Q.copy()
    q[0, 0, 0, 100] = -1.0  # negative density
    sim = _sim(p.with_scheme(Q=q))
    sim.fill_bcs()
    sim.time_step(1e-4)
    f = sim.status()
    assert f & capi.FLAG_NEG_DENSITY
    assert sim.status() == 0  # cleared by the read
    with pytest.raises(capi.McError):
        sim.time_step(-1.0)
    bad = p.with_scheme(ng=1, Q=P.sod_1d(256, ng=1).Q)  # MUSCL needs 2 ghosts
    with pytest.raises(capi.McError):
        _sim(bad)


def test_fp32_form_error_bounds(gpu_lib, oracle_port):
    """FP32 reconstruction/Riemann with FP64 state: relative L1 density error
    against the FP64 oracle stays below 1e-6 on KH after 20 steps."""
    p = P.kelvin_helmholtz_2d(128, seed=1)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(20)
    sim = _sim(p, precision="fp32")
    sim.fill_bcs()
    for dt in ref_dts:
        sim.time_step(dt)
    rho, rho_ref = sim.get_Q()[0], o.get_Q()[0]
    rel_l1 = np.abs(rho - rho_ref).sum() / np.abs(rho_ref).sum()
    assert rel_l1 < 1e-6, rel_l1
    assert sim.status() == 0


@pytest.mark.parametrize("transport", ["hook", "library"])
def test_slab_decomposition_device_loop_single_rank(gpu_lib, oracle_port, transport):
    """The slab path in the device-driven loop (SlabSim.advance) on one rank
    is bit-identical to the reference run of the same periodic problem: the
    Python boundary hook, and the library's own NCCL exchange (one rank
    sending its periodic ghost rows to itself) with the NCCL all-reduce of
    the CFL minimum."""
    from mosscap_b200.distributed import SlabSim
    p = P.kelvin_helmholtz_2d(96, seed=6)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(8)
    s = SlabSim(p, rank=0, world=1, transport=transport)
    s.fill_bcs()
    dts = s.advance(8)
    _assert_same(np.array(dts), ref_dts, "dt")
    _assert_same(s.sim.get_Q(), o.get_Q(), "state")


def test_cfl_reduce_hook(gpu_lib):
    """mc_set_cfl_reduce_hook: called once before every dt of the device loop
    (and by mc_compute_dt), in-stream, on the word the dt is formed from."""
    import ctypes
    import torch
    from mosscap_b200 import capi
    from mosscap_b200.distributed import _CudaArray
    from mosscap_b200.hydro import HydroSim
    p = P.kelvin_helmholtz_2d(64, seed=2)
    base = HydroSim(p)
    base.fill_bcs()
    ref = base.advance(6)
    calls = []

    def count(user, ptr, stream):
        calls.append(ptr)

    sim = HydroSim(p)
    sim.fill_bcs()
    hook = capi.CFL_REDUCE_FN(count)
    capi.check(sim.lib.mc_set_cfl_reduce_hook(sim.ctx, hook, None), "hook")
    dts = sim.advance(6)
    assert len(calls) == 7
    _assert_same(dts, ref, "dt with an identity hook")
    # a hook that caps the minimum: every dt follows the capped value
    cap = 0.5 * ref[0] / p.max_cfl
    cap_bits = int(np.array([cap]).view(np.int64)[0])

    def capper(user, ptr, stream):
        w = torch.as_tensor(_CudaArray(ptr, (1,), "<i8"), device="cuda")
        torch.clamp_(w, max=cap_bits)

    sim2 = HydroSim(p)
    sim2.fill_bcs()
    hook2 = capi.CFL_REDUCE_FN(capper)
    capi.check(sim2.lib.mc_set_cfl_reduce_hook(sim2.ctx, hook2, None), "hook")
    dts2 = sim2.advance(4)
    assert dts2[0] == cap * p.max_cfl and (dts2 <= cap * p.max_cfl).all()
    assert sim2.compute_dt() <= cap * p.max_cfl
    capi.check(sim2.lib.mc_set_cfl_reduce_hook(sim2.ctx, capi.CFL_REDUCE_FN(0), None), "unhook")


@pytest.mark.parametrize("transport", ["hook", "library"])
def test_slab_decomposition_single_rank(gpu_lib, oracle_port, transport):
    """The slab path (y faces filled by the boundary hook or the library's
    exchange, the host-driven loop) on one rank with a self-periodic exchange
    is bit-identical to the reference run of the same periodic problem."""
    from mosscap_b200.distributed import SlabSim
    p = P.kelvin_helmholtz_2d(96, seed=5)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(8)
    s = SlabSim(p, rank=0, world=1, transport=transport)
    s.fill_bcs()
    dts = [s.step() for _ in range(8)]
    _assert_same(np.array(dts), ref_dts, "dt")
    _assert_same(s.sim.get_Q(), o.get_Q(), "state")


def _rel_errors(a, ref):
    d = np.abs(a - ref)
    return float(d.sum() / np.abs(ref).sum()), float(d.max() / np.abs(ref).max())


@pytest.mark.parametrize("n", [64, 128])
def test_sedov_fp64_and_fp32_against_oracle(gpu_lib, oracle_port, n):
    """3D Sedov at 64^3 and 128^3 to t = 0.05: the FP64 form is bit-exact
    against the oracle (dt sequence and state); the FP32 form (its own dt
    sequence from its FP64 state) stays within 1e-7 relative L1 and 1e-5
    relative Linf in density. The errors are printed for the record."""
    p = P.sedov_3d(n)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(10 ** 6)
    ref = o.get_Q()
    out = {}
    for precision in ("fp64", "fp32"):
        sim = _sim(p, precision=precision)
        sim.fill_bcs()
        dts = sim.run(10 ** 6)
        assert sim.time == o.time == 0.05
        q = sim.get_Q()
        if precision == "fp64":
            _assert_same(dts, ref_dts, "dt")
            _assert_same(q, ref, "state")
        ng = p.ng
        core = (slice(None), slice(ng, -ng), slice(ng, -ng), slice(ng, -ng))
        out[precision] = _rel_errors(q[core][0], ref[core][0]) + (len(dts), len(ref_dts))
        assert sim.status() == 0
    print(f"sedov {n}^3 t=0.05 density (rel L1, rel Linf, steps, oracle steps):", out)
    l1, linf = out["fp32"][:2]
    assert l1 < 1e-7 and linf < 1e-5, out


@pytest.mark.parametrize("ndim,n,rec,rs,st", [(1, 700, "muscl", "hllc", "rk2"), (2, 97, "weno5z", "hllc", "ssprk3"),
                                              (3, 35, "ppm", "hll", "ssprk4")])
def test_gravity_source_multi_tile(gpu_lib, oracle_port, ndim, n, rec, rs, st):
    """The gravity source term (source/SourceTerms/Gravity.cpp) on grids of
    several tiles, host and device loops, bit-exact against the oracle."""
    q = P.random_state(ndim, n, n, n, ng=3, seed=77 + ndim)
    p = P.Problem(f"gravity_{ndim}d", ndim, n, n if ndim > 1 else 1, n if ndim > 2 else 1, ng=3, dx=1.0 / n,
                  bc=("wall", "wall", "periodic", "periodic", "zerograd", "symmetricoutflowdiode"),
                  reconstruction=rec, slope_limiter="monotonizedcentral", riemann_solver=rs, time_stepper=st,
                  gamma=1.4, max_cfl=0.5, max_time=1.0, output_delta=0.02, gravity=(0.5, -2.0, 1.0), Q=q)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(12)
    for loop in ("host", "device"):
        sim = _sim(p)
        sim.fill_bcs()
        dts = sim.run(12, device_loop=(loop == "device"))
        _assert_same(dts, ref_dts, f"dt ({loop})")
        _assert_same(sim.get_Q(), o.get_Q(), f"state ({loop})")
        assert sim.status() == 0


@pytest.mark.parametrize("rec,rs", [("ppm", "hll"), ("weno5z", "hllc")])
def test_tracers_3d_multi_tile(gpu_lib, oracle_port, rec, rs):
    """Two passive tracers in 3D on a grid of several x-y tiles and z chunks
    (45 x 38 x 70), host and device loops, bit-exact against the oracle."""
    nx, ny, nz = 45, 38, 70
    q = P.random_state(3, nx, ny, nz, ng=3, num_tracers=2, seed=91)
    p = P.Problem("tracers_3d", 3, nx, ny, nz, ng=3, num_tracers=2, dx=1.0 / nz,
                  bc=("periodic", "periodic", "wall", "zerograd", "symmetric", "symmetricoutflowdiode"),
                  reconstruction=rec, slope_limiter="monotonizedcentral", riemann_solver=rs, time_stepper="ssprk3",
                  gamma=1.4, max_cfl=0.3, max_time=1.0, output_delta=0.02, Q=q)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(5)
    for loop in ("host", "device"):
        sim = _sim(p)
        sim.fill_bcs()
        dts = sim.run(5, device_loop=(loop == "device"))
        _assert_same(dts, ref_dts, f"dt ({loop})")
        _assert_same(sim.get_Q(), o.get_Q(), f"state ({loop})")


@pytest.mark.parametrize("ndim,nx,ny,nz,rec,rs", [(2, 98, 76, 1, "weno5z", "hllc"), (2, 62, 94, 1, "ppm", "hll"),
                                                  (2, 70, 40, 1, "fog", "rusanov"),
                                                  (3, 46, 40, 33, "ppm", "hll"), (3, 40, 36, 31, "weno5z", "hllc")])
def test_tma_tile_path_tile_unaligned(gpu_lib, oracle_port, ndim, nx, ny, nz, rec, rs):
    """Grids whose row length is even (the stage input can be described by a
    tensor map, so the tiled kernels stage their tiles with TMA copies),
    with partial tiles on both axes, boxes that run past the array at the
    upper edges, and wall / diode / zero-gradient faces: host and device
    loops bit-exact against the oracle, FP64."""
    q = P.random_state(ndim, nx, ny, nz, ng=3, seed=5 + nx)
    p = P.Problem(f"tma_{ndim}d", ndim, nx, ny, nz if ndim > 2 else 1, ng=3, dx=1.0 / nx,
                  bc=("wall", "zerograd", "symmetricoutflowdiode", "wall", "zerograd", "symmetric"),
                  reconstruction=rec, slope_limiter="monotonizedcentral", riemann_solver=rs, time_stepper="ssprk3",
                  gamma=1.4, max_cfl=0.3, max_time=1.0, output_delta=0.02, Q=q)
    assert (nx + 6) % 2 == 0
    o = _oracle(oracle_port, p)
    ref_dts = o.run(6)
    for loop in ("host", "device"):
        sim = _sim(p)
        sim.fill_bcs()
        dts = sim.run(6, device_loop=(loop == "device"))
        _assert_same(dts, ref_dts, f"dt ({loop})")
        _assert_same(sim.get_Q(), o.get_Q(), f"state ({loop})")
        assert sim.status() == 0


@pytest.mark.parametrize("loop", ["host", "device"])
def test_z_slab_decomposition_single_rank(gpu_lib, oracle_port, loop):
    """A 3D z slab (PPM + HLL, periodic in z, walls and zero-gradient
    elsewhere) through the library's NCCL exchange of ghost planes, one rank
    sending its periodic planes to itself: bit-identical to the oracle."""
    from mosscap_b200.distributed import SlabSim
    nx, ny, nz = 40, 34, 36
    q = P.random_state(3, nx, ny, nz, ng=3, seed=123)
    p = P.Problem("zslab", 3, nx, ny, nz, ng=3, dx=1.0 / nz,
                  bc=("wall", "zerograd", "symmetric", "wall", "periodic", "periodic"),
                  reconstruction="ppm", slope_limiter="monotonizedcentral", riemann_solver="hll",
                  time_stepper="ssprk3", gamma=1.4, max_cfl=0.3, max_time=1.0, output_delta=0.02, Q=q)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(6)
    s = SlabSim(p, rank=0, world=1, transport="library")
    s.fill_bcs()
    dts = [s.step() for _ in range(6)] if loop == "host" else s.advance(6)
    _assert_same(np.array(dts), ref_dts, "dt")
    _assert_same(s.sim.get_Q(), o.get_Q(), "state")


@pytest.mark.parametrize("nx,ny,nz", [(46, 40, 37), (62, 35, 64)])
def test_fp32_form_3d_tma_tiles_against_oracle(gpu_lib, oracle_port, nx, ny, nz):
    """The FP32 form's 3D z pass stages its tiles with TMA copies (even row
    length, no tracers): tile-unaligned grids with partial x tiles, z chunks
    past the array and wall / zero-gradient / symmetric faces, six SSPRK3
    steps on the FP64 oracle's dt sequence; density within 1e-6 relative
    L1 of the oracle."""
    q = P.random_state(3, nx, ny, nz, ng=3, seed=nx + nz)
    p = P.Problem("fp32_3d", 3, nx, ny, nz, ng=3, dx=1.0 / nx,
                  bc=("wall", "zerograd", "symmetric", "wall", "zerograd", "symmetricoutflowdiode"),
                  reconstruction="ppm", slope_limiter="monotonizedcentral", riemann_solver="hll",
                  time_stepper="ssprk3", gamma=1.4, max_cfl=0.3, max_time=1.0, output_delta=0.02, Q=q)
    assert (nx + 6) % 2 == 0 and nz + 6 >= 36
    o = _oracle(oracle_port, p)
    ref_dts = o.run(6)
    sim = _sim(p, precision="fp32")
    sim.fill_bcs()
    for dt in ref_dts:
        sim.time_step(dt)
    rho, rho_ref = sim.get_Q()[0], o.get_Q()[0]
    rel_l1 = np.abs(rho - rho_ref).sum() / np.abs(rho_ref).sum()
    assert rel_l1 < 1e-6, rel_l1
    assert sim.status() == 0


@pytest.mark.parametrize("ny,st,rec,rs,gravity", [(121, "rk2", "ppm", "hll", None),
                                                  (97, "ssprk3", "weno5z", "hllc", (0.3, -1.0, 0.0)),
                                                  (150, "ssprk4", "muscl", "rusanov", None)])
def test_slab_overlap_single_rank(gpu_lib, oracle_port, ny, st, rec, rs, gravity):
    """A 2D slab whose exchange runs beside the interior tile rows
    (mc_set_slab_overlap, on by default; one rank exchanging with itself
    through the library's NCCL path): bit-identical to the oracle and to the
    same slab with the overlap off, in the device- and host-driven loops,
    with stage timing on (one timed interval per stage). ny = 121 leaves one
    row in the last tile row, fewer than ng, so two tile rows at that end
    write layers that are sent."""
    from mosscap_b200 import capi
    from mosscap_b200.distributed import SlabSim
    nx, steps = 70, 10
    q = P.random_state(2, nx, ny, ng=3, seed=ny)
    p = P.Problem("slab_overlap", 2, nx, ny, ng=3, dx=1.0 / ny,
                  bc=("wall", "zerograd", "periodic", "periodic", "zerograd", "zerograd"),
                  reconstruction=rec, slope_limiter="vanleer", riemann_solver=rs, time_stepper=st, gamma=1.4,
                  max_cfl=0.4, max_time=1e30, output_delta=1e30, gravity=gravity, Q=q)
    o = _oracle(oracle_port, p)
    ref_dts = o.run(steps)
    ref = o.get_Q()
    nst = {"rk2": 2, "ssprk3": 3, "ssprk4": 4}[st]
    for overlap in (1, 0):
        for loop in ("device", "host"):
            s = SlabSim(p, rank=0, world=1, transport="library")
            capi.check(s.sim.lib.mc_set_slab_overlap(s.sim.ctx, overlap), "mc_set_slab_overlap")
            s.fill_bcs()
            s.sim.profile_stages(True)
            dts = s.advance(steps) if loop == "device" else [s.step() for _ in range(steps)]
            ms, n = s.sim.stage_time(0)
            s.sim.profile_stages(False)
            what = f"overlap={overlap} {loop}"
            _assert_same(np.array(dts), ref_dts, f"dt ({what})")
            _assert_same(s.sim.get_Q(), ref, f"state ({what})")
            assert n == steps * nst and ms > 0.0, (what, n, ms)
            assert s.sim.status() == 0
            s.sim.close()


def test_slab_overlap_fp32_form_matches_serial_exchange(gpu_lib):
    """The FP32 compute form through the overlapped slab step (one rank,
    the library's NCCL path): bit-identical to the same slab with the
    overlap off, in the device-driven loop."""
    from mosscap_b200 import capi
    from mosscap_b200.distributed import SlabSim
    p = P.kelvin_helmholtz_2d(128, seed=9).with_scheme(max_time=1e30, output_delta=1e30)
    runs = []
    for overlap in (1, 0):
        s = SlabSim(p, rank=0, world=1, precision="fp32", transport="library")
        capi.check(s.sim.lib.mc_set_slab_overlap(s.sim.ctx, overlap), "mc_set_slab_overlap")
        s.fill_bcs()
        dts = np.array(s.advance(10))
        runs.append((dts, s.sim.get_Q()))
        assert s.sim.status() == 0
        s.sim.close()
    _assert_same(runs[0][0], runs[1][0], "dt")
    _assert_same(runs[0][1], runs[1][1], "state")
