"""mc_time_step_noalloc against mc_time_step, through the C ABI.

mc_time_step_noalloc exists for callers that cannot call cudaMalloc (their
device memory belongs to a pool allocator, or they must not synchronise the
device mid-run): it takes its stage buffers from a fixed 16 MiB static device
array instead of a context. Its results must equal the context-based entry
point's bit for bit, on consecutive calls (the static array keeps the previous
call's contents). This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

from mosscap_b200 import problems as P

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _with_tracer(base, k=0):
    """base plus one passive tracer (a smooth mass fraction times rho)."""
    x = np.arange(base.Q.shape[-1]).reshape(1, 1, 1, -1)
    frac = 0.3 + 0.2 * np.sin(x / (9.0 + k)) * np.ones(base.Q.shape[1:])[None]
    return base.with_scheme(num_tracers=1, Q=np.concatenate([base.Q, frac * base.Q[:1]], axis=0))


CASES = {
    "kh2d_weno_hllc_ssprk3": lambda: (P.kelvin_helmholtz_2d(96, seed=4), "fp64"),
    "sod1d_tracer_rk2": lambda: (_with_tracer(P.sod_1d(512)), "fp64"),
    "sedov3d_ppm_hll_ssprk3": lambda: (P.sedov_3d(24), "fp64"),
    # ssprk4 reuses stage buffer A (Q -> A -> B -> A -> Q)
    "kh2d_muscl_hllc_ssprk4": lambda: (P.kelvin_helmholtz_2d(80, seed=5).with_scheme(
        reconstruction="muscl", slope_limiter="monotonizedcentral", time_stepper="ssprk4"), "fp64"),
    "sedov3d_tracer_ssprk4": lambda: (_with_tracer(P.sedov_3d(20)).with_scheme(time_stepper="ssprk4"), "fp64"),
    # the FP32 compute form on the same static scratch
    "kh2d_weno_hllc_fp32": lambda: (P.kelvin_helmholtz_2d(96, seed=6), "fp32"),
    "sedov3d_ppm_hll_fp32": lambda: (P.sedov_3d(24), "fp32"),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_matches_context_entry_point(gpu_lib, case):
    """Two calls in a row on the shared static scratch, bit for bit against
    the allocating context path (the same kernels with their own buffers)."""
    from mosscap_b200 import capi
    from mosscap_b200.hydro import HydroSim
    lib = gpu_lib
    p, precision = CASES[case]()
    ref = HydroSim(p, precision=precision)  # mc_create + mc_time_step (allocating path)
    ref.fill_bcs()
    q2 = ref.Q.clone()                      # the same filled state for the static path
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        dt = ref.compute_dt()
        ref.time_step(dt)
        st = lib.mc_time_step_noalloc(ctypes.byref(ref._grid), ctypes.byref(ref._scheme),
                                      ctypes.c_void_p(q2.data_ptr()), dt, stream)
        capi.check(st, "mc_time_step_noalloc")
        torch.cuda.synchronize()
        a, b = ref.get_Q(), q2.cpu().numpy()
        assert np.array_equal(_bits(a), _bits(b)), f"call {call}: {np.count_nonzero(_bits(a) != _bits(b))} differ"


@pytest.mark.parametrize("stepper", ["rk2", "ssprk4"])
def test_noalloc_matches_oracle(gpu_lib, oracle_port, stepper):
    """FP64 on the static scratch against the C restatement of the reference
    (two steps with the oracle's own dt), bit for bit."""
    from mosscap_b200 import capi
    from mosscap_b200.hydro import HydroSim
    O = oracle_port
    p = P.kelvin_helmholtz_2d(64, seed=7).with_scheme(time_stepper=stepper)
    o = O.OracleSim(O.OracleConfig(**p.scheme_fields()), "port")
    o.set_Q(p.Q)
    o.fill_bcs()
    sim = HydroSim(p)  # only for its descriptors and a device copy of Q
    q = torch.from_numpy(o.get_Q()).cuda()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        dt = o.compute_dt()
        o.time_step(dt)
        capi.check(gpu_lib.mc_time_step_noalloc(ctypes.byref(sim._grid), ctypes.byref(sim._scheme),
                                                ctypes.c_void_p(q.data_ptr()), dt, stream), "mc_time_step_noalloc")
        torch.cuda.synchronize()
        a, b = o.get_Q(), q.cpu().numpy()
        assert np.array_equal(_bits(a), _bits(b)), f"call {call}: {np.count_nonzero(_bits(a) != _bits(b))} differ"


def test_noalloc_rejects_oversize(gpu_lib):
    from mosscap_b200 import capi
    from mosscap_b200.hydro import HydroSim
    p = P.kelvin_helmholtz_2d(600, seed=0)  # 2 x 4 x 606^2 doubles > 16 MiB
    sim = HydroSim(p)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = gpu_lib.mc_time_step_noalloc(ctypes.byref(sim._grid), ctypes.byref(sim._scheme),
                                      ctypes.c_void_p(sim.Q.data_ptr()), 1e-4, stream)
    assert st == 4  # MC_ERR_OUT_OF_MEMORY
    assert b"16 MiB" in gpu_lib.mc_last_error()
    with pytest.raises(capi.McError):
        capi.check(st, "mc_time_step_noalloc")
