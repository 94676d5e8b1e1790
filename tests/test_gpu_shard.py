"""Block sharding on one GPU: a grid split into shard pools (each with its
own blocks and halo copies) gives the unsharded pool's RBGS solve bit for bit.

Every shard pool lives on the same device, and the halo exchange between
them is a device-to-device copy ordered by the host between passes -- no
kernel waits on another -- so this runs the multi-GPU code path's passes,
exchange lists and gathered sums without a second GPU.  The residual history
(per-block partial sums gathered into global order and added by the pool's
cross-block tree) and every block's pressure must equal the unsharded solve's.
"""
import numpy as np
import pytest
import torch

import ffvgpu
from helpers import VC, assert_bitwise, device_problem, interior, problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level,ranks,count", [(2, 2, 12), (3, 3, 20)])
def test_sharded_rbgs_equals_unsharded(level, ranks, count):
    g, inp, O = problem(level)
    Pg = device_problem(g, inp)
    Pg.fill("X", 0.0)
    ref = Pg.solve_rbgs(1.0, count, 0.0)
    xg = interior(Pg.download("X", VC)).copy()
    fields = {f: Pg.download(f, VC) for f in ("AP", "AW", "AE", "AS", "AN", "AB", "AT", "B")}
    parts = []
    for r in range(ranks):
        S = ffvgpu.Shard(g.desc(), ranks, r)
        P = ffvgpu.Pool(S.desc())
        for f, a in fields.items():
            P.upload(f, a[S.local], VC)
        P.fill("X", 0.0)
        parts.append((P, S))

    def exchange():
        torch.cuda.synchronize()
        views = [ffvgpu.pool_iterate(P, S.owned + S.halo) for P, S in parts]
        for r, (P, S) in enumerate(parts):
            for p, rcv in S.recv.items():
                src = parts[p][1].send[r]
                views[r][torch.as_tensor(rcv, dtype=torch.long, device="cuda")] = \
                    views[p][torch.as_tensor(src, dtype=torch.long, device="cuda")]
        torch.cuda.synchronize()

    def gather(partials):
        out = np.zeros(g.nb)
        for (P, S), part in zip(parts, partials):
            out[S.local[:S.owned]] = part[:S.owned]
        return out

    hist = ffvgpu.sharded_rbgs(parts, 1.0, count, exchange, gather)
    assert_bitwise(hist, ref["history"], "residual history")
    for P, S in parts:
        x = interior(P.download("X", VC))
        assert_bitwise(x[:S.owned], xg[S.local[:S.owned]], f"pressure of shard {S.rank}")
        P.close()
    Pg.close()
