"""Where the recipes that read the reference checkout (the host build of its kernels, the golden-vector and save-file
generators, the reference arm's install) find it: the directory named by $ISW_REFERENCE, else a directory named
``reference`` beside this repository. ``reference_root()`` is None when neither holds the reference's sources; callers
then skip the step. Test infrastructure only."""
import os
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]


def reference_root():
    cand = os.environ.get('ISW_REFERENCE')
    p = Path(cand) if cand else REPO.parent / 'reference'
    return p if (p / 'src' / 'insilica' / 'kernels').is_dir() else None


def reference_kernels():
    r = reference_root()
    return None if r is None else r / 'src' / 'insilica' / 'kernels'
