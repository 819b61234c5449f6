"""Per-component L1 error between two states (pure numpy; loads no library).

The rule every accuracy figure of this package uses (tests, smoke, bench), over interior cells of
ghosted (9, ny + 2 ng, nx + 2 ng) states in the reference's component order (rho, mx, my, mz, E,
bx, by, bz, psi):

* rho, m_x, m_y, m_z, E, B_x, B_y, B_z: relative L1, sum|a - b| / sum|b|, or the absolute
  sum|a - b| where b is identically zero (m_z and B_z of a 2D state with v_z = B_z = 0 and no
  Hall term stay exactly zero);
* psi: sum|a - b| / max(sum|b|, c_h * sum|B|). psi carries the divergence error of B at the GLM
  speed c_h (its flux is c_h^2 B_n and B_n's flux is psi), so c_h |B| is its natural scale. On
  smooth, nearly divergence-free states psi starts at zero and stays at the rounding level of that
  scale, where sum|b| alone would measure rounding rather than agreement; where psi is large
  (shocked states) the rule is the plain relative L1.

With ``vector_scale`` (the rule of the FP32-mixed bar) the components of the momentum and the
magnetic field are held on their vector's scale: sum|a_c - b_c| / sum|b_vec| with |b_vec| the
Euclidean norm of m (for m_x, m_y, m_z) or of B (for B_x, B_y, B_z) per cell. A component that is
a small part of its vector is then held to the accuracy of the vector, not of itself: with a Hall
term, B_z and m_z are generated from zero by a second derivative of B (the curl of
eta_H J x B / |B|, J itself a difference of B), which FP32 differencing at fine grids resolves only
to about eps_FP32 / (k dx)^2 relative to B_z itself.
"""

from __future__ import annotations

import numpy as np

COMPONENTS = ("rho", "mx", "my", "mz", "energy", "bx", "by", "bz", "psi")


def component_l1(a: np.ndarray, b: np.ndarray, c_h: float, ng: int = 2,
                 vector_scale: bool = False) -> np.ndarray:
    """L1 error of a against b per component (9 values), by the rule above."""
    ai = a[:, ng:a.shape[1] - ng, ng:a.shape[2] - ng]
    bi = b[:, ng:b.shape[1] - ng, ng:b.shape[2] - ng]
    num = np.empty(9)
    den = np.empty(9)
    for c in range(9):  # one component at a time: no full-size temporaries of all nine
        num[c] = float(np.abs(ai[c] - bi[c]).sum())
        den[c] = float(np.abs(bi[c]).sum())
    bmag = float(np.sqrt(bi[5] * bi[5] + bi[6] * bi[6] + bi[7] * bi[7]).sum())
    den[8] = max(den[8], float(c_h) * bmag)
    if vector_scale:
        mmag = float(np.sqrt(bi[1] * bi[1] + bi[2] * bi[2] + bi[3] * bi[3]).sum())
        den[1:4] = mmag
        den[5:8] = bmag
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)
