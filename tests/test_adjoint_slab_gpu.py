"""The discrete adjoint split into y slabs (mc_adjoint_set_slab_*) against
the single-domain adjoint, on a 64^2 periodic Kelvin-Helmholtz problem over
8 SSPRK3 steps with checkpoints every 3 steps and a random cotangent of the
final state (so that every step's dt sensitivity is nonzero).

One rank (its own periodic neighbour), through the library's NCCL exchange
and through the hook: forward state, initial-state cotangent and dJ/dgamma
equal the single domain's bit for bit, since the tiles, the per-tile partial
sums and their order are the same.

Two and four ranks on one GPU, each a process with the hook staged through
host memory (gloo; no kernel waits on another rank: every exchange is a
host-side collective between launches): the forward state equals the single
domain's bit for bit. The sums of the dt and gamma sensitivities run over
other partitions, so the cotangents differ from the single domain's by
rounding, and at t = 0 rounding is not a small effect in every direction:
the KH bands are flat to rounding in density, x velocity and pressure, where
the WENO-Z weights' derivatives are ratios of rounding-level smoothness
indicators, so the initial-state cotangent's components along those fields
are rounding noise of the size of the cotangent itself (in the single domain
too: its own reverse step from t = 0 maps two cotangents 1e-11 apart to
results 3 apart). The comparison is therefore made where the derivative is
defined: dJ/d(vy field) and dJ/dgamma of the KH initial condition
(adjoint.kh_initial_state), whose perturbations keep those fields fixed,
within 1e-10 of the largest."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from mosscap_b200 import problems as P

pytestmark = pytest.mark.gpu

N = 64
STEPS = 8
CKPT = 3
REL = 1e-10


def _inputs(device="cuda"):
    p = P.kelvin_helmholtz_2d(N, seed=3)
    ng = p.ng
    q0 = torch.tensor(p.Q[:, 0, ng:-ng, ng:-ng], dtype=torch.float64, device=device)
    g = torch.Generator().manual_seed(11)
    w = torch.randn(4, N, N, generator=g, dtype=torch.float64).to(device)
    return p, q0, w


def _single_domain(p, q0, w):
    from mosscap_b200.adjoint import _Runner, pad_periodic
    ng = p.ng
    runner = _Runner(p, p.gamma, CKPT)
    qpad = pad_periodic(q0, ng)
    runner.forward(qpad, STEPS)
    lam = torch.zeros_like(qpad)
    lam[:, 0, ng:-ng, ng:-ng] = w
    dg = runner.backward(lam)
    torch.cuda.synchronize()
    return (qpad[:, 0, ng:-ng, ng:-ng].cpu().numpy(), lam[:, 0, ng:-ng, ng:-ng].cpu().numpy(), dg)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


@pytest.mark.parametrize("transport", ["library", "hook"])
def test_adjoint_single_rank_slab_matches_single_domain(gpu_lib, transport):
    from mosscap_b200.adjoint import SlabAdjoint
    p, q0, w = _inputs()
    qf_ref, lam_ref, dg_ref = _single_domain(p, q0, w)
    adj = SlabAdjoint(p, p.gamma, 0, 1, CKPT, transport=transport)
    qf = adj.forward(adj.rows(q0), STEPS)
    lam, dg = adj.backward(adj.rows(w))
    torch.cuda.synchronize()
    assert np.array_equal(_bits(qf.cpu().numpy()), _bits(qf_ref))
    assert np.array_equal(_bits(lam.cpu().numpy()), _bits(lam_ref)), \
        f"max |diff| {np.abs(lam.cpu().numpy() - lam_ref).max()}"
    assert np.float64(dg).view(np.uint64) == np.float64(dg_ref).view(np.uint64), (dg, dg_ref)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir, errors):
    import torch.distributed as dist
    from mosscap_b200.adjoint import SlabAdjoint
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        p, q0, w = _inputs()
        adj = SlabAdjoint(p, p.gamma, rank, world, CKPT, transport="host")
        qf = adj.forward(adj.rows(q0), STEPS)
        lam, dg = adj.backward(adj.rows(w))
        torch.cuda.synchronize()
        np.save(os.path.join(out_dir, f"q{rank}.npy"), qf.cpu().numpy())
        np.save(os.path.join(out_dir, f"l{rank}.npy"), lam.cpu().numpy())
        np.save(os.path.join(out_dir, f"g{rank}.npy"), np.array([dg]))
    except Exception as e:  # reported to the parent
        errors.put(f"rank {rank}: {type(e).__name__}: {e}")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_adjoint_slab_ranks_on_one_gpu_match_single_domain(gpu_lib, world, tmp_path):
    ctx = mp.get_context("spawn")
    errors = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), errors)) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=300)
    for pr in procs:
        if pr.is_alive():
            pr.kill()
    msgs = []
    while not errors.empty():
        msgs.append(errors.get())
    assert not msgs, msgs
    assert all(pr.exitcode == 0 for pr in procs), [pr.exitcode for pr in procs]

    p, q0, w = _inputs()
    qf_ref, lam_ref, dg_ref = _single_domain(p, q0, w)
    qf = np.concatenate([np.load(os.path.join(tmp_path, f"q{r}.npy")) for r in range(world)], axis=1)
    lam = np.concatenate([np.load(os.path.join(tmp_path, f"l{r}.npy")) for r in range(world)], axis=1)
    dgs = [float(np.load(os.path.join(tmp_path, f"g{r}.npy"))[0]) for r in range(world)]
    assert np.array_equal(_bits(qf), _bits(qf_ref)), "forward state differs from the single domain"
    # every rank holds the same summed dJ/dgamma of the dynamics
    assert all(np.float64(d).view(np.uint64) == np.float64(dgs[0]).view(np.uint64) for d in dgs), dgs
    gv, gg = _through_initial_condition(p, lam, dgs[0])
    gv_ref, gg_ref = _through_initial_condition(p, lam_ref, dg_ref)
    scale = np.abs(gv_ref).max()
    assert np.abs(gv - gv_ref).max() <= REL * scale, np.abs(gv - gv_ref).max() / scale
    assert abs(gg - gg_ref) <= REL * abs(gg_ref), (gg, gg_ref)


def _through_initial_condition(p, lam0, dgamma):
    """(dJ/d(vy field), dJ/dgamma) for the initial state
    kh_initial_state(vy, gamma) given the initial-state cotangent lam0 and
    the dynamics' dJ/dgamma."""
    from mosscap_b200.adjoint import kh_initial_state, kh_vy
    vy = torch.tensor(kh_vy(p), device="cuda").requires_grad_(True)
    g = torch.tensor(p.gamma, dtype=torch.float64, device="cuda", requires_grad=True)
    q0 = kh_initial_state(vy, g, p)
    gv, gg = torch.autograd.grad(q0, (vy, g), torch.tensor(lam0, device="cuda"))
    return gv.cpu().numpy(), gg.item() + dgamma
