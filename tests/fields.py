"""Per-field error measures used by the parity tests.

Fields are the conserved variables rho, rho u, rho v, rho w, E and, with SST,
k and omega.  Each field's error is taken relative to the size of its own
field, except the three momentum components, which are taken relative to the
momentum vector's size: a component that is identically small (rho w of a
planar vortex) would otherwise turn rounding into a large relative error.
"""

import numpy as np

NAMES = ("rho", "rho_u", "rho_v", "rho_w", "E")


def _np(a):
    if hasattr(a, "detach"):
        a = a.detach().double().cpu().numpy()
    return np.asarray(a, dtype=np.float64)


def per_field(a, b):
    """{field: (relative L2, relative max)} of state a against reference b
    ((..., >=5) conserved columns; extra columns are ignored)."""
    a, b = _np(a), _np(b)
    d = a[..., :5] - b[..., :5]
    mom = b[..., 1:4]
    out = {}
    for v, name in enumerate(NAMES):
        ref = mom if 1 <= v <= 3 else b[..., v]
        l2 = float(np.linalg.norm(d[..., v]) / max(np.linalg.norm(ref), 1e-300))
        mx = float(np.max(np.abs(d[..., v])) / max(np.max(np.abs(ref)), 1e-300))
        out[name] = (l2, mx)
    return out


def scalar(a, b):
    """(relative L2, relative max) of a scalar field a against b."""
    a, b = _np(a), _np(b)
    d = a - b
    return (float(np.linalg.norm(d) / max(np.linalg.norm(b), 1e-300)),
            float(np.max(np.abs(d)) / max(np.max(np.abs(b)), 1e-300)))


def worst(errs, which=1):
    """Largest of the per-field errors (which = 0: L2, 1: max)."""
    return max(v[which] for v in errs.values())
