"""Golden vectors for the cross-correlation misfit and the station-coordinate conversion.

FIXTURE-GENERATION INFRASTRUCTURE ONLY (runs where the reference tree exists):

    python tests/golden/make_misc_golden.py

* ``xcorr.npz``: the reference's own ``Elastic3D.computeResidualCrossCorrelation`` and
  ``computeCostFunctionCrossCorrelation`` (mainPropElastic3D_MT.py:2145-2209), imported
  unmodified through ``ref_harness`` and called on seeded gathers (with an all-zero
  observed trace, an all-zero modelled trace and an orthogonal pair to reach every guard).
* ``stations.npz``: the station latitude/longitude strings of
  LecturaEstacionesSismologicasProyecto/lecturaEstacionesSismologicasProyecto.py (read as
  literals with ``ast``, the script is not executed) and the grid positions the reference
  stored from them (npyFiles/rec_pos_{x,y,z}.npy).
"""
from __future__ import annotations

import ast
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_harness  # noqa: E402


class _G:
    def __init__(self, vx, vy, vz):
        self.Vx, self.Vy, self.Vz = vx, vy, vz


def xcorr_golden():
    main, _ = ref_harness.import_reference()
    rng = np.random.default_rng(21)
    nt, nrec = 57, 9
    obs = [rng.standard_normal((nt, nrec)).astype(np.float32) for _ in range(3)]
    mod = [(0.7 * o + 0.3 * rng.standard_normal((nt, nrec))).astype(np.float32) for o in obs]
    obs[0][:, 2] = 0.0                      # zero observed trace
    mod[1][:, 4] = 0.0                      # zero modelled trace
    mod[2][:, 6] = 0.0
    obs[2][:, 6] = 0.0                      # both zero: dot guard too
    res = [np.zeros((nt, nrec), np.float32) for _ in range(3)]
    me = types.SimpleNamespace(obsGather=_G(*obs), modGather=_G(*mod), resGather=_G(*res),
                               LenStations=nrec, costFunction=[], totalCostFunction=0.0)
    main.Elastic3D.computeResidualCrossCorrelation(me)
    main.Elastic3D.computeCostFunctionCrossCorrelation(me, 0)
    np.savez_compressed(os.path.join(HERE, "xcorr.npz"), obs=np.stack(obs), mod=np.stack(mod),
                        res=np.stack([me.resGather.Vx, me.resGather.Vy, me.resGather.Vz]),
                        cost=np.float64(me.totalCostFunction))


def stations_golden():
    d = os.path.join(ref_harness.REF_DIR, "LecturaEstacionesSismologicasProyecto")
    with open(os.path.join(d, "lecturaEstacionesSismologicasProyecto.py"), encoding="utf-8") as f:
        tree = ast.parse(f.read())
    lit = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and isinstance(node.value, ast.Constant):
            for t in node.targets:
                if isinstance(t, ast.Name) and t.id in ("latitud_1", "longitud_1"):
                    lit[t.id] = node.value.value
    out = {k: np.load(os.path.join(d, "npyFiles", f"rec_pos_{k}.npy")) for k in "xyz"}
    np.savez_compressed(os.path.join(HERE, "stations.npz"), latitude=np.array(lit["latitud_1"]),
                        longitude=np.array(lit["longitud_1"]), rec_x=out["x"], rec_y=out["y"],
                        rec_z=out["z"])


if __name__ == "__main__":
    xcorr_golden()
    stations_golden()
