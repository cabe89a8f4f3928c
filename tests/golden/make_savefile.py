"""Write tests/golden/save_ref.zip with the REFERENCE's own save writer (src/insilica/io/save.py, imported from the
reference checkout): fixed meta and arrays, so tests can check that isw.savefile writes the same bytes and reads it.

    python tests/golden/make_savefile.py [--ref <reference checkout>]
"""
import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def content():
    i = np.arange(3 * 50, dtype=np.float64).reshape(3, 50)
    return dict(level=4, name='fixture', dt=1800.0), dict(h=np.sin(i), u=np.cos(i[:2]), theta=290.0 + i[:1], n=np.arange(7))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=None)
    a = ap.parse_args()
    if a.ref is None:
        sys.path.insert(0, str(HERE.parents[1]))
        from oracle import refpath
        a.ref = refpath.reference_root()
        if a.ref is None:
            sys.exit('make_savefile: reference checkout not found (pass --ref or set ISW_REFERENCE)')
    sys.path.insert(0, str(Path(a.ref) / 'src'))
    from insilica.io import save
    meta, arrays = content()
    save.write(HERE / 'save_ref.zip', meta, arrays)
    print('save_ref.zip', (HERE / 'save_ref.zip').stat().st_size, 'bytes')


if __name__ == '__main__':
    main()
