"""Operation counts of the refinement passes (the roofline numerators):
smb_batch_count_refine_ops re-runs the fast-mode f32 refinement with its
field evaluations' operations counted, smb_batch_count_exact_ops the exact
one.  The counts are deterministic, the re-run leaves the edge results as
they were, and the warm start, which saves evaluations, counts fewer."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_refine_op_counts_are_stable_and_leave_results():
    from sesmesh_b200 import native, warm_start, workloads
    from sesmesh_b200 import surface as S
    g = workloads.globule330()
    p = S.SurfaceParams.ses(1.4).with_spacing(0.25).with_refine("fast")
    eng = S.SurfaceEngine(g["spheres"], p)
    mlp = native.Mlp(eng.dev, warm_start.load())
    eng.set_warm_start(mlp)
    eng.run_device()
    before = eng.mesh()
    pos0 = before.positions.copy()
    plain = [eng.count_refine_ops() for _ in range(2)]
    warm = [eng.count_refine_ops(mlp) for _ in range(2)]
    assert plain[0] == plain[1] > 0
    assert warm[0] == warm[1] > 0
    assert warm[0] < plain[0]
    after = eng.mesh()
    assert np.array_equal(after.positions, pos0)
    before.close(), after.close()
    eng.close()


def test_exact_op_counts_are_stable():
    from sesmesh_b200 import workloads
    from sesmesh_b200 import surface as S
    g = workloads.globule330()
    eng = S.SurfaceEngine(g["spheres"], S.SurfaceParams.ses(1.4).with_spacing(0.25))
    eng.run_device()
    a, b = eng.count_exact_ops(), eng.count_exact_ops()
    assert a == b > 0
    eng.close()
