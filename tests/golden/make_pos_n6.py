"""Write tests/golden/pos_n6.npz: the level-6 generator positions smoothed by the REFERENCE's own Lloyd iteration
(``insilica.grid.icosa.lloyd_scvt``, unchanged, imported from the reference checkout, run with NumPy on the host to its
1e-11 rad tolerance), in the icosphere's (v1) numbering, with the iteration count and the last move.

The reference runs this step with CuPy from level 6 up (``grid/__init__.py:26``, "results differ only by rounding");
its NumPy form takes about ten minutes at level 6 on a few host cores, so the result is kept as a fixture.
``oracle/build_ref.py`` builds the reference's level-6 grid from it with the reference's own geometry, renumbering and
TRiSK code (the grid the CPU reference arm of the benchmark runs on). Run from the repository root:

    python tests/golden/make_pos_n6.py [--ref <reference checkout>]
"""
import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=None)
    ap.add_argument('--level', type=int, default=6)
    a = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    from oracle import refpath
    ref = Path(a.ref) if a.ref else refpath.reference_root()
    if ref is None:
        sys.exit('make_pos_n6: reference checkout not found (pass --ref or set ISW_REFERENCE)')
    sys.path.insert(0, str(ref / 'src'))
    from insilica.grid import icosa
    t = time.time()
    V, faces = icosa.icosphere(a.level)
    adj, deg = icosa._adjacency(faces, V.shape[0])
    ring = icosa._sorted_ring(V, adj, deg)
    with np.errstate(invalid='ignore', divide='ignore'):      # pentagon pad slots are degenerate and masked
        pos, iters, moved = icosa.lloyd_scvt(V, ring, deg, xp=np, max_iters=200000)
    out = HERE / f'pos_n{a.level}.npz'
    np.savez_compressed(out, pos=pos, lloydIters=np.int64(iters), lloydMoved=np.float64(moved), level=np.int64(a.level))
    print(out.name, out.stat().st_size, 'bytes;', iters, 'iterations, last move', moved, f'{time.time() - t:.0f} s')


if __name__ == '__main__':
    main()
