"""The slab decomposition end to end with two ranks on one GPU.

Two processes (gloo process group, both on cuda:0) each advance one y slab
of a 64^2 periodic Kelvin-Helmholtz problem through SlabSim: ghost rows
after every stage through the boundary hook and the global CFL minimum
through the CFL reduce hook, both staged through host memory. No kernel
waits on the other rank: every exchange is a host-side collective between
launches. The slabs' interiors, stacked, and the dt sequence must equal the
single-domain run of the C restatement of the reference bit for bit, in the
host-driven loop (compute_dt / time_step) and in the device-driven loop
(mc_advance with the hooks called in-stream)."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

STEPS = 8
N = 64


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, loop, out_dir, errors):
    import torch
    import torch.distributed as dist
    from mosscap_b200 import problems as P
    from mosscap_b200.distributed import SlabSim
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        p = P.kelvin_helmholtz_2d(N, seed=3)
        slab = SlabSim(p, rank, world, device=torch.device("cuda", 0), transport="host")
        slab.fill_bcs()
        if loop == "host":
            dts = np.array([slab.step() for _ in range(STEPS)])
        else:
            dts = np.asarray(slab.advance(STEPS))
        np.save(os.path.join(out_dir, f"q{rank}.npy"), slab.interior())
        np.save(os.path.join(out_dir, f"dt{rank}.npy"), dts)
        status = slab.sim.status()
        if status:
            errors.put(f"rank {rank}: status flags {status}")
    except Exception as e:  # reported to the parent
        errors.put(f"rank {rank}: {type(e).__name__}: {e}")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("loop", ["host", "device"])
def test_two_slab_ranks_on_one_gpu_match_single_domain(gpu_lib, oracle_port, loop, tmp_path):
    from mosscap_b200 import problems as P
    world = 2
    ctx = mp.get_context("spawn")
    errors = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, loop, str(tmp_path), errors)) for r in range(world)]
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

    O = oracle_port
    p = P.kelvin_helmholtz_2d(N, seed=3)
    ref = O.OracleSim(O.OracleConfig(**p.scheme_fields()), "port")
    ref.set_Q(p.Q)
    ref.fill_bcs()
    rdts = ref.run(STEPS)
    ng = p.ng
    qref = ref.get_Q()[:, :, ng:-ng, ng:-ng]
    q = np.concatenate([np.load(os.path.join(tmp_path, f"q{r}.npy")) for r in range(world)], axis=2)
    for r in range(world):
        dts = np.load(os.path.join(tmp_path, f"dt{r}.npy"))
        assert np.array_equal(dts.view(np.uint64), rdts.view(np.uint64)), f"rank {r}: dt sequence differs"
    assert np.array_equal(q.view(np.uint64), qref.view(np.uint64)), \
        f"{np.count_nonzero(q.view(np.uint64) != qref.view(np.uint64))} interior values differ"
