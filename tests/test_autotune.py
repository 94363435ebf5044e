"""Launch-shape autotuner: cache handling on CPU, tuning of a small batch on the GPU."""
import os

import numpy as np
import pytest

from conftest import rel_err


class _FakeBatch:
    def __init__(self, grids):
        self.specs = [dict(nx=a, ny=b, nz=c, lenpml=w) for a, b, c, w in grids]


def test_cache_roundtrip_and_key_order(tmp_path):
    from elastic_fm_vp_vs_rho_b200 import autotune
    p = str(tmp_path / "sub" / "tune.json")
    assert autotune.load_cache(p) == {}
    k1 = autotune.batch_key(_FakeBatch([(64, 64, 48, 10), (32, 40, 24, 5)]))
    k2 = autotune.batch_key(_FakeBatch([(32, 40, 24, 5), (64, 64, 48, 10)]))
    assert k1 == k2  # instance order does not matter
    autotune.save_cache({k1: {"rows": 1, "ychunk": 8, "ms": 1.5}}, p)
    assert autotune.load_cache(p)[k1]["rows"] == 1
    with open(p, "w") as f:
        f.write("{not json")
    assert autotune.load_cache(p) == {}


def test_candidates_cover_both_tile_heights_and_ring_depths():
    from elastic_fm_vp_vs_rho_b200 import autotune
    rows = {r for r, _, _ in autotune.DEFAULT_CANDIDATES}
    rings = {(r, d) for r, d, _ in autotune.DEFAULT_CANDIDATES}
    assert rows == {1, 2} and (1, 6) in rings and (2, 6) not in rings
    assert all(0 <= yc <= 64 for _, _, yc in autotune.DEFAULT_CANDIDATES)


@pytest.mark.gpu
def test_tune_applies_a_choice_and_reuses_the_cache(golden_c1scale, cuda, tmp_path):
    from elastic_fm_vp_vs_rho_b200 import ShotBatch, autotune
    d = golden_c1scale
    cp = np.concatenate([d[k] for k in ("ax", "bx", "ay", "by", "az", "bz")]).astype(np.float32)
    b = ShotBatch()
    b.add(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]), lenpml=int(d["lenpml"]),
          dx=float(d["dx"]), dt=float(d["dt"]), nt=int(d["nt"]), cpml=cp, lam=d["lam_true"],
          mu=d["mu_true"], rho=d["rho_true"], wavelet=d["waveform"], src=[d["src"][0]],
          mt=[d["mt_mod"]], rec=np.stack([d["rec_x"], d["rec_y"], d["rec_z"]], axis=1))
    ref = b.forward().cpu().numpy()
    p = str(tmp_path / "tune.json")
    c1 = autotune.tune(b, nt_probe=12, path=p, repeats=1,
                       candidates=((2, 4, 0), (1, 4, 0), (1, 6, 8)))
    assert not c1["cached"] and c1["rows"] in (1, 2) and os.path.exists(p)
    got = b.forward().cpu().numpy()
    assert rel_err(got, ref) < 1e-5  # any launch shape computes the same gathers
    c2 = autotune.tune(b, path=p)
    assert c2["cached"] and (c2["rows"], c2["ychunk"]) == (c1["rows"], c1["ychunk"])
