"""GPU tests of the potential gradients (pdmk_evaluate_grad_double), plain FP64
path, against the Ewald gradient (oracle.ewald_targets_grad, pinned by finite
differences on the CPU).  Bars, relative L2 over all components and max error
max|g - g_ref| / max|g_ref|: 1e-4 at 6 digits, 1e-7 at 9, 1e-10 at 12 (the
potential's own bars are 2e-6, 2e-9, 2e-12; the gradient of the residual and
plane-wave expansions loses about one to two digits).  Each case prints a
"PARITY {...}" line with the figures."""
import json

import numpy as np
import pytest

import oracle
import periodicdmk_b200 as pd
from conftest import TRICLINIC, clustered_system, rel_l2, uniform_system

pytestmark = pytest.mark.gpu

SWAPPED = np.array([[0.8, 0.1, 0.0], [0.0, 1.3, 0.2], [0.0, 0.0, 1.0]])  # longest vector not first: rotated frame


def _max_err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("system", ["cube", "clustered_triclinic", "swapped_axes"])
@pytest.mark.parametrize("nd,bar", [(6, 1e-4), (9, 1e-7), (12, 1e-10)])
def test_gradient_vs_ewald(system, nd, bar):
    if system == "cube":
        cell, pos, q = uniform_system(3000, 71)
        npl = 30
    elif system == "clustered_triclinic":
        cell, pos, q = clustered_system(3000, 72, TRICLINIC, n_clusters=4, sigma=0.03)
        npl = 30
    else:
        cell, pos, q = uniform_system(2000, 73, SWAPPED)
        npl = 25
    t = pd.PeriodicDMKTree(cell, pos, n_digits=nd, n_per_leaf=npl, nz=4)
    pot, grad = t.evaluate_grad(q)
    pot_plain = t.evaluate(q)
    t.close()
    assert rel_l2(pot, pot_plain) < 1e-13
    ref_pot, ref_grad = oracle.ewald_targets_grad(cell, pos, q, np.arange(len(q)), s=6.5)
    e, m = rel_l2(grad.ravel(), ref_grad.ravel()), _max_err(grad, ref_grad)
    print("PARITY " + json.dumps({"case": "gradient %s %d digits" % (system, nd), "rel_l2_vs_ewald": e,
                                  "max_err_vs_ewald": m, "pot_rel_l2_vs_ewald": rel_l2(pot, ref_pot)}))
    assert e < bar and m < bar * 10


def test_gradient_errors():
    cell, pos, q = uniform_system(200, 74)
    tf = pd.PeriodicDMKTree(cell, pos, 6, 30, 4, precision="float")
    with pytest.raises(ValueError):
        tf.evaluate_grad(q)
    tf.close()
    assert pd.library().pdmk_evaluate_grad_double(None, 0, None, None, None, None) == -1
