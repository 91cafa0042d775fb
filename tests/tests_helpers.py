"""Diagnostics shared by the tests (same definitions as tests/golden/gen_golden.py)."""
import numpy as np


def domain_means(st) -> np.ndarray:
    """[th, qc, qr, surface rain, kinetic energy] over interior cells; kinetic
    energy is 0.5 rhou (u^2 + w^2) at the stored points."""
    f = st.fields
    inner = (slice(1, -1), slice(1, -1))
    rhou = st.prof["rhou"][None, 1:-1]
    ke = 0.5 * rhou * (f["u"][inner] ** 2 + f["w"][inner] ** 2)
    return np.array([f["th"][inner].mean(), f["qc"][inner].mean(), f["qr"][inner].mean(),
                     st.precip[1:-1].mean(), ke.mean()])
