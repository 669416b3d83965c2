"""Array names, padded shapes and periodic fills of the serial-periodic lane.

The names, their order and the padded C-order (z, y, x) shapes are the
reference operator API's (src/cm1core/cuda_sound3_periodic.py:51-99,449-503;
src/cm1core/cuda_psolver3_trajectory.py:93-126), so dictionaries built for the
reference launchers can be passed here unchanged.  The order is also the
field order of ``gm1b_periodic_arrays`` in ``include/gm1b.h``.
"""

from __future__ import annotations

import numpy as np

SCALAR_NAMES = (
    "mh", "rr0", "rf0", "c1", "c2", "mf", "piadv", "ppterm", "thv", "ppten",
    "ppi", "pp3d", "ppx", "ppd", "qk", "pk1", "pk2", "mm", "fpk", "divh",
    "hadvp", "elim_c", "elim_d", "tri_aa", "tri_bb", "tri_cc", "tri_dd",
    "tri_pivot", "tri_residual",
)
W_NAMES = ("wten", "wa", "w3d", "rrw")
U_NAMES = ("ua", "u3d", "uten", "rru")
V_NAMES = ("va", "v3d", "vten", "rrv")
METRIC_NAMES = ("dtu0", "dtv0", "uf", "vf", "uh", "vh")
SOUND_ARRAY_NAMES = SCALAR_NAMES + W_NAMES + U_NAMES + V_NAMES + METRIC_NAMES
EXTRA_ARRAY_NAMES = (
    "pi0", "rho0", "rrf0", "th0", "rth0", "tha", "th3d", "sadv", "thten", "divx",
)
ALL_ARRAY_NAMES = SOUND_ARRAY_NAMES + EXTRA_ARRAY_NAMES

# Acoustic scratch arrays whose reference-semantics values are written only
# with GM1B_FLAG_SCRATCH_OUTPUTS (src/cm1core/cuda_sound3_periodic.py:122-147).
SCRATCH_OUTPUT_NAMES = (
    "fpk", "divh", "hadvp", "elim_c", "elim_d", "tri_aa", "tri_bb", "tri_cc",
    "tri_dd", "tri_pivot", "tri_residual",
)

# Outputs of the acoustic operator compared word for word
# (src/cm1core/cuda_sound3_periodic.py:122-147).
SOUND_COMPARE_NAMES = (
    "u3d", "v3d", "w3d", "pp3d", "ppx", "ppd", "rru", "rrv", "rrw", "qk",
    "pk1", "pk2", "mm", "fpk", "divh", "hadvp", "elim_c", "elim_d", "tri_aa",
    "tri_bb", "tri_cc", "tri_dd", "tri_pivot", "tri_residual",
)

# Outputs of the dry trajectory compared word for word
# (src/cm1core/cuda_psolver3_trajectory.py:106-129).
TRAJECTORY_STATE_NAMES = (
    "ua", "u3d", "va", "v3d", "wa", "w3d", "ppi", "pp3d", "ppx", "tha", "th3d",
    "sadv", "rru", "rrv", "rrw", "uten", "vten", "wten", "thten", "divx",
    "tri_pivot", "tri_residual",
)


def _check_dims(ni: int, nj: int, nk: int) -> None:
    for name, value in (("ni", ni), ("nj", nj), ("nk", nk)):
        if isinstance(value, bool) or not isinstance(value, int) or value < 3:
            raise ValueError(f"{name} must be an integer >= 3")


def scalar_shape_zyx(ni: int, nj: int, nk: int) -> tuple[int, int, int]:
    _check_dims(ni, nj, nk)
    return nk + 2, nj + 2, ni + 2


def array_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    """Shapes of the acoustic-stage arrays."""
    scalar = scalar_shape_zyx(ni, nj, nk)
    shapes: dict[str, tuple[int, ...]] = {name: scalar for name in SCALAR_NAMES}
    shapes.update({name: (nk + 2, nj, ni) for name in W_NAMES})
    shapes.update({name: (nk + 2, nj + 2, ni + 1) for name in U_NAMES})
    shapes.update({name: (nk + 2, nj + 1, ni + 2) for name in V_NAMES})
    shapes.update(
        {
            "dtu0": (nj + 2, ni + 1),
            "dtv0": (nj + 1, ni + 2),
            "uf": (ni + 2,),
            "vf": (nj + 2,),
            "uh": (ni + 2,),
            "vh": (nj + 2,),
        }
    )
    return shapes


def trajectory_array_shapes(ni: int, nj: int, nk: int) -> dict[str, tuple[int, ...]]:
    """Shapes of every trajectory array (acoustic arrays plus extras)."""
    shapes = array_shapes(ni, nj, nk)
    scalar = scalar_shape_zyx(ni, nj, nk)
    shapes.update({name: scalar for name in EXTRA_ARRAY_NAMES})
    return shapes


def default_periodic_face_weights(ni: int, nj: int) -> tuple[np.ndarray, np.ndarray]:
    """CM1 serial-periodic face time-step weights: one on live faces, zero on
    the halo rows (u) / columns (v) (src/cm1core/cuda_sound3_periodic.py:494-503)."""
    _check_dims(ni, nj, 3)
    dtu0 = np.zeros((nj + 2, ni + 1), dtype=np.float32)
    dtv0 = np.zeros((nj + 1, ni + 2), dtype=np.float32)
    dtu0[1 : nj + 1, :] = np.float32(1.0)
    dtv0[:, 1 : ni + 1] = np.float32(1.0)
    return dtu0, dtv0


def fill_periodic_scalar_inplace(value: np.ndarray, *, ni: int, nj: int, nk: int) -> None:
    """Periodic halo fill of a padded scalar on levels 1..nk: x halos first,
    then whole y halo rows (so corners wrap in both directions)."""
    for k in range(1, nk + 1):
        value[k, :, 0] = value[k, :, ni]
        value[k, :, ni + 1] = value[k, :, 1]
        value[k, 0, :] = value[k, nj, :]
        value[k, nj + 1, :] = value[k, 1, :]


def fill_periodic_uv_inplace(u: np.ndarray, v: np.ndarray, *, ni: int, nj: int, nk: int) -> None:
    """Periodic halo rows of u and halo columns of v on levels 1..nk."""
    u[1 : nk + 1, 0, :] = u[1 : nk + 1, nj, :]
    u[1 : nk + 1, nj + 1, :] = u[1 : nk + 1, 1, :]
    v[1 : nk + 1, :, 0] = v[1 : nk + 1, :, ni]
    v[1 : nk + 1, :, ni + 1] = v[1 : nk + 1, :, 1]


def zeros_like_shapes(shapes: dict[str, tuple[int, ...]]) -> dict[str, np.ndarray]:
    return {name: np.zeros(shape, dtype=np.float32) for name, shape in shapes.items()}
