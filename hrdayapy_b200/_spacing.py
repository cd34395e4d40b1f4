"""voxel_size="from_geometry" resolution (same contract as the reference's
hrdayapy/_spacing_resolve.py:24-73)."""
from __future__ import annotations

import numpy as np

FROM_GEOMETRY = "from_geometry"


def resolve_voxel_size(voxel_size, anatomy=None, *, param_name: str = "voxel_size") -> float:
    if isinstance(voxel_size, str):
        if voxel_size.strip().lower() != FROM_GEOMETRY:
            raise ValueError(f"Unrecognised {param_name}={voxel_size!r}; the only accepted "
                             f"string value is \"{FROM_GEOMETRY}\" (or pass a float directly).")
        if anatomy is None or "spacing_mm" not in anatomy:
            raise ValueError(f"{param_name}=\"{FROM_GEOMETRY}\" requires the anatomy dict "
                             "(anatomy=...) with a 'spacing_mm' entry.")
        spacing = np.asarray(anatomy["spacing_mm"], dtype=np.float64).ravel()
        if spacing.size > 1 and not np.allclose(spacing, spacing[0]):
            raise ValueError(f"anatomy['spacing_mm']={spacing} is anisotropic, but {param_name} "
                             f"here must be a single isotropic value -- pass a float explicitly.")
        return float(spacing[0])
    return float(voxel_size)
