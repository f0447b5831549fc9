"""Systems of the batched workload (512 Laplacian systems, seed 4) whose
rank cap is too small for tol 1e-8: the reference algorithm (the FP64
oracle of amen_solve2) stalls above the tolerance as well, so a batched
solve that stops short of 1e-8 on them follows the reference, not a fault
of the device path.  CPU only."""
import numpy as np

from oracle.amen import amen_solve2
from oracle.tt import TT, TTMatrix, tt_randn, true_residual
from ttgpu import workloads


def test_small_rank_cap_stalls_in_the_oracle():
    As, ys, rmaxs, shapes = workloads.batch_systems(count=512, seed=4)
    i = 32  # d = 7, n = 64, rmax = 9
    assert shapes[i] == (7, 64, 9) and rmaxs[i] == 9
    A, y = As[i], ys[i]
    Ao = TTMatrix.from_flat(A.n, A.m, A.r, A.core)
    yo = TT.from_flat(y.n, y.r, y.core)
    x0 = tt_randn([int(v) for v in A.n], A.d, 2, np.random.default_rng(i))
    x, info = amen_solve2(Ao, yo, 1e-8, x0, None, rmax=rmaxs[i], nswp=20)
    assert info["sweeps"] == 20
    assert min(info["max_res"]) > 1e-6  # stalls two orders above the tolerance
    assert max(x.r) <= rmaxs[i] + 4      # rank cap plus the kick rank
    assert true_residual(Ao, x, yo) > 1e-8
