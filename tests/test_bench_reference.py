"""The benchmark's reference arm runs the reference's own kernels (oracle/_ref, built for the host) on the reference's
own level-6 grid and loads nothing of isw's device library; its line describes the same workload (`config`) as the
isw arm's."""
import json
import subprocess
import sys

import pytest

from conftest import ROOT

SCRIPT = r'''
import json, sys
sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3']
sys.path.insert(0, {root!r})
import bench
bench.main()
maps = open('/proc/self/maps').read()
print(json.dumps({{'libisw_loaded': 'libisw.so' in maps, 'ref_loaded': 'libref_kernels.so' in maps}}))
'''


def test_reference_arm_loads_no_isw_device_code():
    from oracle import build_ref, refkernels
    if not (refkernels.available() and build_ref.grid_path(6).exists()):
        pytest.skip('oracle/_ref (the reference kernels and grid built for the host) is not present')
    r = subprocess.run([sys.executable, '-c', SCRIPT.format(root=str(ROOT))], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith('{')]
    line, maps = lines[0], lines[-1]
    assert line['impl'] == 'reference' and line['value'] > 0 and 'unavailable' not in line
    assert maps == {'libisw_loaded': False, 'ref_loaded': True}
    sys.path.insert(0, str(ROOT))
    import bench

    class A:
        level = 6
    from isw import grid as G
    g = G.load(build_ref.grid_path(6))
    assert line['config'] == bench.member_config(A, g, 1)     # the dict the isw arm prints for the same run
