"""Independent solves of different operators in one graph launch
(cpsgpu_solve_batch): every solve gives the iteration count and solution of
its own DiracOp::InvCg run alone, two of them on one lattice (their
reductions must not share buffers), in FP64 and mixed precision."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpMobius, DiracOpWilson, Lattice, gen_gauge, gen_gaussian, solve_batch
from helpers import rel

pytestmark = pytest.mark.gpu


def _lat(L, seed):
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=seed))
    return lat


def test_solve_batch_matches_single_solves():
    A.check(A.lib().cpsgpu_set_device(0))
    la, lb, lc = _lat((4, 4, 4, 8), 701), _lat((8, 8, 8, 8), 702), _lat((4, 4, 4, 4), 703)
    ops = [DiracOpDwf(la, mass=0.01, ls=8), DiracOpDwf(la, mass=0.1, ls=8),  # one lattice, two masses
           DiracOpWilson(lb, mass=1 / (2 * 0.12) - 4), DiracOpMobius(lc, mass=0.05, ls=6)]
    for prec in (A.DOUBLE, A.SINGLE):
        srcs = [gen_gaussian(D.f_size, seed=710 + k) for k, D in enumerate(ops)]
        single = []
        for D, b in zip(ops, srcs):
            x = np.zeros(D.f_size)
            r = D.InvCg(x, b, stop_rsd=1e-10, precision=prec)
            single.append((x, r))
        sols = [np.zeros(D.f_size) for D in ops]
        res = solve_batch(list(zip(ops, sols, srcs)), stop_rsd=1e-10, precision=prec)
        for (x1, r1), x, r in zip(single, sols, res):
            assert r.status == A.CONVERGED and r.true_res <= 1e-10
            assert r.iterations == r1.iterations
            assert rel(x, x1) < 1e-12
    with pytest.raises(A.CpsGpuError):  # one operator twice in one precision
        solve_batch([(ops[0], np.zeros(ops[0].f_size), srcs[0]), (ops[0], np.zeros(ops[0].f_size), srcs[0])])
