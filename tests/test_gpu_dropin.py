"""The reference's own command-line driver, relinked against libgrappolo_b200.so.

oracle/Makefile builds Grappolo's driverForGraphClustering.cpp twice from its
sources: driver_ref with every reference object (the reference program) and
driver_b200 with the same driver object, loaders and utilities but with the
library in place of the clustering, colouring, coarsening, vertex-following,
comparison and binary-file objects (driverForGraphClustering.cpp:163-189 calls
runMultiPhaseColoring / runMultiPhaseBasic through their C++ signatures).  Both
run `-f 9 -c <c> -m 1000 -d 1e-4 -t 1e-6 -o` at OMP_NUM_THREADS=1 on the same
binary graph file; the community files they write must be equal byte for byte
and they must print the same final modularity and cluster count.  `-c 2`
(balanced recolouring) runs against driver_ref_vbase, driver_ref with the one
missing `return` of vBaseRedistribution added, on graphs where the function's
first-fit scan stays inside its arrays (tests/golden/vbase.npz).
"""
import os
import re
import shutil
import subprocess

import pytest

from grappolo_b200 import graphs
from _golden import vbase_cases

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DROPIN = os.path.join(os.path.dirname(HERE), 'oracle', '_ref', 'dropin')
REF_BIN = os.path.join(DROPIN, 'driver_ref')
REF_VBASE_BIN = os.path.join(DROPIN, 'driver_ref_vbase')
B200_BIN = os.path.join(DROPIN, 'driver_b200')


def _run(binary, graph_file, args):
    env = dict(os.environ, OMP_NUM_THREADS='1')
    p = subprocess.run([binary, '-f', '9', graph_file, *args, '-o'], env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, (binary, p.returncode, p.stdout[-2000:], p.stderr[-2000:])
    with open(graph_file + '_clustInfo', 'rb') as f:
        clusters = f.read()
    mod = re.search(r'Final modularity\s*:\s*(-?[\d.]+)', p.stdout)
    ncl = re.search(r'Final number of clusters\s*:\s*(\d+)', p.stdout)
    assert mod and ncl, p.stdout[-2000:]
    return clusters, mod.group(1), int(ncl.group(1))


def _graph_file(tmp_path, name):
    path = str(tmp_path / f'{name}.bin')
    if name == 'karate':
        shutil.copy(os.path.join(HERE, 'golden', 'karate.bin'), path)
    elif name == 'planted_100k':
        graphs.write_binary(graphs.planted_partition(), path)
    elif name == 'planted_100k_w':
        graphs.write_binary(graphs.random_weights(graphs.planted_partition()), path)
    elif name == 'rmat14':
        graphs.write_binary(graphs.rmat(14, seed=9), path)
    else:
        graphs.write_binary({c[0]: c[1] for c in vbase_cases()}[name], path)
    return path


@pytest.mark.skipif(not all(os.path.exists(b) for b in (REF_BIN, REF_VBASE_BIN, B200_BIN)),
                    reason='drop-in drivers not built (oracle/Makefile dropin)')
@pytest.mark.parametrize('name,coloring', [('karate', '1'), ('planted_100k', '1'),
                                           ('planted_100k_w', '1'), ('rmat14', '1'),
                                           ('karate', '0'), ('planted_100k', '0'),
                                           ('sc3000', '2'), ('sc6000', '2'), ('sc30000', '2')])
def test_driver_relinked_against_library(tmp_path, name, coloring):
    args = ['-c', coloring, '-m', '1000', '-d', '0.0001', '-t', '0.000001']
    ref_dir, b200_dir = tmp_path / 'ref', tmp_path / 'b200'
    ref_dir.mkdir()
    b200_dir.mkdir()
    src = _graph_file(tmp_path, name)
    ref_file, b200_file = str(ref_dir / 'g.bin'), str(b200_dir / 'g.bin')
    shutil.copy(src, ref_file)
    shutil.copy(src, b200_file)
    c_ref, q_ref, n_ref = _run(REF_VBASE_BIN if coloring == '2' else REF_BIN, ref_file, args)
    c_b200, q_b200, n_b200 = _run(B200_BIN, b200_file, args)
    assert c_b200 == c_ref
    assert q_b200 == q_ref
    assert n_b200 == n_ref
