"""Generate tests/golden/numba_cuda_b200.npz: the reference's own Numba-CUDA
horizon march run on a B200.

Run on a machine with a B200 and the reference installed under
``baseline/_ref`` (``baseline/load_reference.py`` imports it and opens its
CUDA import gate to numba's built-in CUDA target):

    python tests/golden/make_numba_golden.py [--out DIRECTORY]

Case: the plain configuration's 512 x 512 DEM at 20 m (seed 1) as the
primary DEM and the 2000 x 2000 regional DEM at 240 m (seed 1002) around
it; the centred tile (column 192, row 192), observer 1.5 m above the
terrain, the public 1,000 km range (capped per DEM by the reference's
segment builder), 1440 azimuths.  Segments come from the reference's host
builder (``geometry.build_subpatch_segments_numba``), pyramids from the
reference session's ``build_max_pyramid``, slopes from its
``subpatch_hierarchical_all_passes`` (``cuda_backend.py:1445-1552``).  Stored
for 12 azimuths (every 120th): the segments of those azimuths and the slopes
of all 16,384 pixels at them, with the device name and numba's version.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "baseline"))

AZIMUTHS = np.arange(0, 1440, 120)
TILE = dict(tile_column=192, tile_row=192, tile_width=128, tile_height=128, subpatch_size=8)
OBSERVER_M = 1.5


def main() -> None:
    import argparse

    import numba

    parser = argparse.ArgumentParser()
    parser.add_argument("--out", default=str(HERE))
    args = parser.parse_args()

    import load_reference
    from lunarscout_b200 import synthetic

    load_reference.import_reference(enable_numba_cuda=True)
    from lunarscout._numba_horizon import cuda_backend, geometry

    def reference_dem(ours):
        projection = geometry.ProjectionParameters.from_array(ours.projection.as_array())
        return geometry.DemGrid(ours.elevation_m, np.array(ours.geo_transform, dtype=np.float64),
                                projection)

    dems = [reference_dem(synthetic.config1_dem()), reference_dem(synthetic.regional_dem())]
    values, _centers, _convergence = geometry.build_subpatch_segments_numba(
        dems, tile_column=TILE["tile_column"], tile_row=TILE["tile_row"],
        tile_width=TILE["tile_width"], azimuth_count=1440, maximum_distance_m=1_000_000.0,
        observer_elevation_m=OBSERVER_M, subpatch_size=8,
        grid_convergence=geometry.GridConvergenceInput(0.0, 0.0, 0.0), parallel=True)
    session = cuda_backend.CudaSession(device_id=0)
    pyramids = [session.build_max_pyramid(dem) for dem in dems]
    slopes, _ = session.subpatch_hierarchical_all_passes(values, pyramids,
                                                         observer_elevation_m=OBSERVER_M, **TILE)
    target = Path(args.out) / "numba_cuda_b200.npz"
    np.savez_compressed(
        target,
        azimuths=AZIMUTHS.astype(np.int32),
        segments=np.ascontiguousarray(values[AZIMUTHS], dtype=np.float32),
        slopes=np.ascontiguousarray(slopes[:, AZIMUTHS], dtype=np.float32),
        tile=np.array([TILE["tile_column"], TILE["tile_row"]], dtype=np.int32),
        observer_elevation_m=np.float32(OBSERVER_M),
        device=np.array(session.info.name), numba=np.array(numba.__version__),
    )
    print("wrote", target, session.info)


if __name__ == "__main__":
    main()
