"""Save files in the reference's format (reference src/insilica/io/save.py:14-34): an uncompressed zip holding
`meta.json` (sorted keys, indent 1, with formatVersion and the sorted array names) and one `.npy` per array, every
entry stamped 1980-01-01 00:00:00 and written in sorted order, so the same state always gives the same bytes and
either project reads the other's files."""
import io
import json
import zipfile

import numpy as np

FORMAT_VERSION = 1
STAMP = (1980, 1, 1, 0, 0, 0)


def write(path, meta, arrays):
    names = sorted(arrays)
    head = dict(meta, formatVersion=FORMAT_VERSION, arrays=names)
    with zipfile.ZipFile(path, 'w', compression=zipfile.ZIP_STORED) as z:
        z.writestr(zipfile.ZipInfo('meta.json', date_time=STAMP), json.dumps(head, sort_keys=True, indent=1))
        for name in names:
            raw = io.BytesIO()
            np.lib.format.write_array(raw, np.ascontiguousarray(arrays[name]), allow_pickle=False)
            z.writestr(zipfile.ZipInfo(name + '.npy', date_time=STAMP), raw.getvalue())


def read(path):
    """(meta, {name: array}); refuses other format versions."""
    with zipfile.ZipFile(path) as z:
        meta = json.loads(z.read('meta.json'))
        if meta.get('formatVersion') != FORMAT_VERSION:
            raise ValueError(f'save file format {meta.get("formatVersion")}, expected {FORMAT_VERSION}')
        arrays = {n: np.lib.format.read_array(io.BytesIO(z.read(n + '.npy')), allow_pickle=False) for n in meta['arrays']}
    return meta, arrays
