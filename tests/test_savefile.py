"""Save files in the reference's format (no GPU): isw.savefile writes the same bytes as the reference's own writer
(tests/golden/save_ref.zip, made by tests/golden/make_savefile.py with the reference's io/save.py) and reads them back;
a different format version is refused."""
import importlib.util
import json
import zipfile

import numpy as np
import pytest

from conftest import GOLDEN


def fixture_content():
    spec = importlib.util.spec_from_file_location('make_savefile', GOLDEN / 'make_savefile.py')
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.content()


def test_same_bytes_as_reference(tmp_path):
    from isw import savefile
    meta, arrays = fixture_content()
    savefile.write(tmp_path / 'ours.zip', meta, arrays)
    assert (tmp_path / 'ours.zip').read_bytes() == (GOLDEN / 'save_ref.zip').read_bytes()
    m2, a2 = savefile.read(GOLDEN / 'save_ref.zip')
    assert m2['level'] == 4 and m2['arrays'] == sorted(arrays)
    for k, v in arrays.items():
        assert np.array_equal(a2[k], v) and a2[k].dtype == v.dtype


def test_other_version_refused(tmp_path):
    from isw import savefile
    p = tmp_path / 'v2.zip'
    with zipfile.ZipFile(p, 'w') as z:
        z.writestr('meta.json', json.dumps(dict(formatVersion=2, arrays=[])))
    with pytest.raises(ValueError):
        savefile.read(p)
