"""Failure detection in the batched Anderson solve.

The reference stops the whole program when an iteration fails
(src/iterate_mod.fp.f90:412-420).  Here every instance carries a status word
computed on the device from its iteration's reductions (<dev, dev> and
max |dev|), so an instance whose fields turn non-finite is retired on its
own while the others go on.  The fault is injected on the host: a NaN in
one instance's initial field."""
import numpy as np
import pytest

from pscf_b200.engine import Engine, FP64, MIXED
from tests.cases import diblock, lamellar_guess

pytestmark = pytest.mark.gpu


def _systems(n):
    return [diblock(1, [32], "lamellar", [1.7], fA=0.5, chiN=15.0) for _ in range(n)]


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_nan_instance_retired_while_others_converge(prec):
    ss = _systems(3)
    w = np.stack([lamellar_guess(s) for s in ss])
    clean = Engine(_systems(1), FP64)
    _, _, ref = clean.iterate_am(w[:1], error_max=1e-9, max_itr=400)
    clean.close()
    w[1, 0, 5] = np.nan
    e = Engine(ss, prec)
    _, _, res = e.iterate_am(w, error_max=1e-9, max_itr=400)
    e.close()
    assert res[1]["status"] == "nonfinite" and not res[1]["converged"], res[1]
    for i in (0, 2):
        assert res[i]["converged"] and res[i]["status"] == "converged", res[i]
        assert abs(res[i]["f_helmholtz"] - ref[0]["f_helmholtz"]) < 1e-9


def test_status_words_maxiter_and_running():
    ss = _systems(2)
    w = np.stack([lamellar_guess(s) for s in ss])
    e = Engine(ss, FP64)
    e.am_begin(w, error_max=1e-12, max_itr=3)
    e.am_iterate(2)
    _, _, mid = e.am_results(want_fields=False)
    assert all(r["status"] == "running" for r in mid)
    while e.am_iterate(5) > 0:
        pass
    _, _, res = e.am_results(want_fields=False)
    e.close()
    assert all(r["status"] == "maxiter" and not r["converged"] for r in res)
