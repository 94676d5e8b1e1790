"""The precision form's outer loop: defect correction against BiCGSTAB (CPU).

A precision form can also be built as RB-SOR sweeps inside an FP64
defect-correction loop.  The oracle restates that loop (orc_mixed_dc: r = b -
A x in FP64, e = the mixed form's RB-SOR preconditioner applied to r, x += e)
with the same preconditioner as the mixed BiCGSTAB form.  On the sphere grid
it converges far too slowly to be the product form: this test records that,
for 32-bit and for FP64 data alike, which is why the GPU form keeps the
BiCGSTAB recurrence around the same preconditioner.
"""
import numpy as np

from helpers import problem


def test_defect_correction_stalls_where_bicgstab_converges():
    g, inp, O = problem(1)
    O.field("X")[...] = 0.0
    dc = O.solve_mixed_dc(1.5, 8, 4, 300, 1e-8)
    O.field("X")[...] = 0.0
    dc64 = O.solve_mixed_dc(1.5, 8, 4, 300, 1e-8, fp64_data=True)
    O.field("X")[...] = 0.0
    bi = O.solve_mixed(1.5, 8, 4, 300, 1e-8)
    # BiCGSTAB around the same preconditioner: 1e-8 within a hundred iterations
    assert bi["status"] == 0 and bi["count"] <= 100 and bi["residual"] <= 1e-8
    # defect correction: 300 corrections (2400 sweeps) leave the residual
    # above 1e-3, decreasing monotonically but slowly ...
    for r in (dc, dc64):
        h = r["history"]
        assert r["count"] == 301 and len(h) == 300
        assert h[-1] > 1e-3 and np.all(np.diff(h) < 0)
    # ... and the 32-bit data are not the cause: FP64 data give the same
    # history to three digits
    assert np.allclose(dc["history"], dc64["history"], rtol=1e-3)
