"""The data-parallel material fit on CPU: two gloo ranks with different
gradients end every step with identical parameters, equal to one process
stepping with the mean gradient (raymotion_b200.inverse.MaterialFit)."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _setup(n_mat=16):
    g = torch.Generator().manual_seed(3)
    lo = torch.tensor([0.05, 0.05, 0.05, 0.05, 0.0, 0.0, 0.0, 1.3])
    hi = torch.tensor([0.95, 0.95, 0.95, 1.0, 20.0, 20.0, 20.0, 1.7])
    true = lo + (hi - lo) * torch.rand(n_mat, 8, generator=g)
    mask = torch.rand(n_mat, 8, generator=g) < 0.7
    start = torch.where(mask, lo + (hi - lo) * torch.rand(n_mat, 8, generator=g), true)
    grads = [torch.randn(3, n_mat * 8, generator=g) for _ in range(2)]  # per rank, 3 steps
    return start, true, mask, lo, hi, grads


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from raymotion_b200.inverse import MaterialFit
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        start, true, mask, lo, hi, grads = _setup()
        fit = MaterialFit(start, true, mask, lo, hi)
        for k in range(3):
            fit.step(grads[rank][k])
        out.put((rank, fit.params().numpy()))
    finally:
        dist.destroy_process_group()


def test_two_rank_fit_equals_mean_gradient_fit():
    from raymotion_b200.inverse import MaterialFit
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(q.get(timeout=5) for _ in range(2))
    start, true, mask, lo, hi, grads = _setup()
    ref = MaterialFit(start, true, mask, lo, hi)
    for k in range(3):
        ref.step((grads[0][k] + grads[1][k]) / 2)
    assert (got[0] == got[1]).all()
    assert torch.allclose(torch.from_numpy(got[0]), ref.params(), rtol=0, atol=1e-6)
    # the fitted entries moved, the others did not
    assert not torch.allclose(ref.params()[mask], start[mask])
    assert torch.equal(ref.params()[~mask], true[~mask])


def test_single_process_step_matches_manual_adam():
    from raymotion_b200.inverse import MaterialFit
    start, true, mask, lo, hi, grads = _setup()
    fit = MaterialFit(start, true, mask, lo, hi, lr=0.05)
    g = grads[0][0]
    fit.step(g)
    # first Adam step: u -= lr * sign(grad) (bias-corrected m/sqrt(v) = +-1)
    u0 = (start - lo) / (hi - lo)
    gu = torch.where(mask, g.view(16, 8) * (hi - lo), torch.zeros_like(u0))
    expect = torch.where(mask, lo + (hi - lo) * (u0 - 0.05 * torch.sign(gu)).clamp(0, 1), true)
    assert torch.allclose(fit.params(), expect, atol=1e-5)
