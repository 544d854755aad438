"""Parity metrics between device results and the FP64 oracle.

The tolerance of the engine's FP32/FP64 mixed path against the FP64
restatement of the reference is 1e-5 relative on every cell mass and on
every barycentre (normalised by the domain extent, 1000), with the volume
of the smallest resolvable piece as the mass floor."""
import numpy as np

SUCCESS = 4
MASS_RTOL = 1e-5
BARY_TOL = 1e-5


def compare(got, got_status, ref, ref_status, mass_floor=1e-3):
    """got/ref: (n,4) (m*x, m*y, m*z, m).  Returns a dict of metrics."""
    both = (got_status == SUCCESS) & (ref_status == SUCCESS)
    m, mr = got[:, 3], ref[:, 3]
    denom = np.maximum(np.abs(mr), mass_floor)
    rel = np.abs(m - mr) / denom
    rel = rel[both]
    nz = both & (np.abs(mr) > mass_floor) & (np.abs(m) > mass_floor)
    bary = np.zeros(0)
    if nz.any():
        b = got[nz, :3] / m[nz, None]
        br = ref[nz, :3] / mr[nz, None]
        bary = np.abs(b - br).max(1) / 1000.0
    nonempty = (np.abs(m) > mass_floor) & (got_status == SUCCESS)
    nonempty_ref = (np.abs(mr) > mass_floor) & (ref_status == SUCCESS)
    return {
        "n": len(m),
        "status_mismatch": int((got_status != ref_status).sum()),
        "nonempty_symdiff": int((nonempty != nonempty_ref).sum()),
        "mass_max_rel": float(rel.max()) if rel.size else 0.0,
        "mass_rms_rel": float(np.sqrt((rel ** 2).mean())) if rel.size else 0.0,
        "bary_max": float(bary.max()) if bary.size else 0.0,
        "bary_rms": float(np.sqrt((bary ** 2).mean())) if bary.size else 0.0,
        "total_rel": float(abs(m[both].sum() - mr[both].sum()) / max(abs(mr[both].sum()), 1e-300)),
    }


def assert_parity(metrics, mass_rtol=MASS_RTOL, bary_tol=BARY_TOL):
    assert metrics["status_mismatch"] == 0, metrics
    assert metrics["nonempty_symdiff"] == 0, metrics
    assert metrics["mass_max_rel"] <= mass_rtol, metrics
    assert metrics["bary_max"] <= bary_tol, metrics
