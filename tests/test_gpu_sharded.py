"""Slot-sharded loop on the CUDA path (run on a B200): ranks that each hold
Nb = Nred/ntasks bosonic slots, exchanging Phi(R), Sigma_V and max|F_r| over
gloo, reproduce the loop of one unsharded context.  The ranks share one GPU;
nothing but host-side collectives links them, so no kernel waits on another
rank."""
from __future__ import annotations

import datetime
import multiprocessing as mp
import socket

import numpy as np
import pytest

from oracle import tups_oracle as O
import parity

pytestmark = pytest.mark.gpu

ITERS = 4
TOL = 1e-12


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, case, out_dir):
    import torch.distributed as dist
    from tups_b200 import Solver
    from tups_b200.sharded import TorchExchange
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        p = parity.to_solver_params(O.Params(f_damping=0.5, ite_max=10, **case))
        sol = Solver(p, 0, rank, world, TorchExchange(0))
        conv = [sol.iteration(i) for i in range(ITERS)]
        np.savez(f"{out_dir}/rank{rank}.npz", sigma=sol.Sigma, slot0=sol.slot0, Nb=sol.Nb,
                 F=np.stack([sol.F(r) for r in "dmst"]), G=np.stack([sol.G(r) for r in "dmst"]),
                 fmax=np.array([[c[f"F_{r}_max"] for r in "dmst"] for c in conv]),
                 mu=np.array([c["mu"] for c in conv]))
        sol.close()
    finally:
        dist.destroy_process_group()


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("case,world", [
    (dict(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2), 2),    # Nred 24: 12 slots per rank
    (dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=12, neighbours=2), 4),   # Nred 36: 9 slots, ranks split a momentum
], ids=["nl5_2ranks", "nl5_4ranks_split_q"])
def test_sharded_loop_matches_unsharded(gpu_lib, tmp_path, case, world):
    from tups_b200 import Solver
    ctx = mp.get_context("spawn")
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, case, str(tmp_path))) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=600)
    assert all(p.exitcode == 0 for p in ps), [p.exitcode for p in ps]

    sol = Solver(parity.to_solver_params(O.Params(f_damping=0.5, ite_max=10, **case)))
    conv = [sol.iteration(i) for i in range(ITERS)]
    F = np.stack([sol.F(r) for r in "dmst"])
    G = np.stack([sol.G(r) for r in "dmst"])
    fmax = np.array([[c[f"F_{r}_max"] for r in "dmst"] for c in conv])
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        s0, nb = int(d["slot0"]), int(d["Nb"])
        assert (s0, nb) == (r * sol.Nb // world, sol.Nb // world)
        assert _rel(d["sigma"], sol.Sigma) < TOL
        assert _rel(d["F"], F[..., s0:s0 + nb]) < TOL
        assert _rel(d["G"], G[..., s0:s0 + nb]) < TOL
        assert _rel(d["fmax"], fmax) < TOL
        assert np.max(np.abs(d["mu"] - np.array([c["mu"] for c in conv]))) < 1e-12
    sol.close()


def test_sharded_rejects_uneven_split(gpu_lib):
    from tups_b200 import Solver, TupsError
    p = parity.to_solver_params(O.Params(Nx=4, Nf=8, neighbours=1))  # Nred = 24
    with pytest.raises(TupsError):
        Solver(p, 0, 0, 5, exchange=lambda *a: None)
