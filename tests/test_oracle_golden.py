"""The CPU oracle against its committed golden fixtures (tests/golden/cases.npz,
written by tests/golden/make_golden.py): the numpy restatement
(oracle/letkf_oracle.py) and the C restatement (oracle/letkf_ref.c through
oracle/cref.py) both reproduce every stored case.

Tolerances: nobsl and PF resampling indices exactly equal; analyses and the
stored W / wvec at sampled points within 1e-12 relative (FP64 both sides;
the C restatement sums in a different order)."""
import numpy as np
import pytest

from oracle import cref
from oracle import letkf_oracle as O
from tests._util import GOLDEN_CASES, field_relerr, load_golden

TOL = 1e-12


def _points(flat, nij1):
    return [(int(q) // nij1, int(q) % nij1) for q in flat]


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_numpy_oracle_reproduces_golden(name):
    d = load_golden(name)
    p, g, ob = d["params"], d["grid"], d["obs"]
    nij1 = g["lon1"].size
    wpts = _points(d["w_points"], nij1)
    spts = _points(d["src_points"], nij1) if "src_points" in d else []
    r = O.da_main(p, g, ob, d["fcst3d"], d["fcst2d"], uniforms=d.get("uniforms"), keep=wpts + spts)
    assert np.array_equal(r.nobsl, d["nobsl"])
    assert field_relerr(r.anal3d, d["anal3d"]) <= TOL
    assert field_relerr(r.anal2d, d["anal2d"]) <= TOL
    for j, q in enumerate(wpts):
        assert np.abs(r.wmat[q] - d["wmat"][j]).max() <= TOL * max(1.0, np.abs(d["wmat"][j]).max())
        assert np.abs(r.wvec[q] - d["wvec"][j]).max() <= TOL * max(1.0, np.abs(d["wmat"][j]).max())
    for j, q in enumerate(spts):
        assert np.array_equal(np.asarray(r.src[q]).astype(np.int16), d["src"][j])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_c_restatement_reproduces_golden(name):
    d = load_golden(name)
    p, g, ob = d["params"], d["grid"], d["obs"]
    rc = cref.da_main(p, g, ob, d["fcst3d"], d["fcst2d"], uniforms=d.get("uniforms"), rsize=8, want_src=True)
    assert int(rc["status"]) == 0
    assert np.array_equal(rc["nobsl"], d["nobsl"])
    assert field_relerr(rc["anal3d"], d["anal3d"]) <= TOL
    assert field_relerr(rc["anal2d"], d["anal2d"]) <= TOL
    if "src_points" in d:
        assert np.array_equal(rc["src"][d["src_points"]].astype(np.int16), d["src"])
