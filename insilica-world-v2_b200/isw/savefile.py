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
    """(meta, {name: array}) of a save file; a file written in another format version is refused (ValueError) before
    any array is decoded."""
    with zipfile.ZipFile(path) as archive:
        meta = json.loads(archive.read('meta.json'))
        found = meta.get('formatVersion')
        if found != FORMAT_VERSION:
            raise ValueError(f'{path}: this reader takes format version {FORMAT_VERSION} only, the file has {found!r}')
        members = {}
        for name in meta['arrays']:
            with archive.open(name + '.npy') as f:
                members[name] = np.lib.format.read_array(io.BytesIO(f.read()), allow_pickle=False)
    return meta, members
