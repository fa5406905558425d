"""The C ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import os
import re
import subprocess

import pytest

from grappolo_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_c_functions():
    text = open(os.path.join(ROOT, 'include', 'grappolo_b200.h')).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(glv_[a-z0-9_]+)\s*\(', text)))


def _exports():
    out = subprocess.run(['nm', '-D', '--defined-only', _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if ' T ' in line}


def test_library_loads():
    L = _lib.lib()
    assert L.glv_version().startswith(b'grappolo_b200')


def test_every_declared_c_entry_point_is_exported():
    names = _declared_c_functions()
    assert len(names) >= 15
    missing = [n for n in names if n not in _exports()]
    assert not missing, missing


# Mangled names of the reference's own objects (g++ Itanium ABI), so code built
# against Grappolo's headers links against this library unchanged.
REFERENCE_SYMBOLS = [
    '_Z21runMultiPhaseColoringP5graphPliiilddii',
    '_Z30algoLouvainWithDistOneColoringP5graphPliPiiddPdS2_',
    '_Z18runMultiPhaseBasicP5graphPlilddii',
    '_Z21parallelLouvianMethodP5graphPliddPdPi',
    '_Z32algoDistanceOneVertexColoringOptP5graphPiiPd',
    '_Z28renumberClustersContiguouslyPll',
    '_Z22buildNextLevelGraphOptP5graphS0_Plli',
    '_Z15vertexFollowingP5graphPl',
    '_Z15buildNewGraphVFP5graphS0_Pll',
    '_Z27algoColoringMultiHashMaxMinP5graphPiiPdii',
    '_Z11removeEdgesllP4edge',
    '_Z19SortEdgesUndirectedllP4edgeS0_Pl',
    '_Z20SortNodeEdgesByIndexlP4edgeS0_Pl',
    '_Z23parse_EdgeListBinaryNewP5graphPc',
    '_Z25writeGraphBinaryFormatNewP5graphPcl',
    '_Z27computeCommunityComparisonsRSt6vectorIlSaIlEElS2_l',
    '_Z22computeGiniCoefficientPli',
    '_Z19vBaseRedistributionP5graphPiii',
]


def test_reference_cxx_api_exported():
    ex = _exports()
    missing = [s for s in REFERENCE_SYMBOLS if s not in ex]
    assert not missing, missing


def test_compat_header_matches_reference_mangling(tmp_path):
    """Compiling against include/grappolo_compat.h produces the same symbol
    names the reference's objects define."""
    src = tmp_path / 'use.cpp'
    src.write_text('#include "grappolo_compat.h"\n'
                   'void use(graph *g, long *c, int *col, double *t, int *it, graph *o) {\n'
                   '  runMultiPhaseColoring(g, c, 1, 16, 0, 1000, 1e-6, 1e-4, 1, 1);\n'
                   '  algoLouvainWithDistOneColoring(g, c, 1, col, 4, -1, 1e-4, t, it);\n'
                   '  runMultiPhaseBasic(g, c, 0, 1000, 1e-6, 1e-4, 1, 1);\n'
                   '  parallelLouvianMethod(g, c, 1, -1, 1e-6, t, it);\n'
                   '  algoDistanceOneVertexColoringOpt(g, col, 1, t);\n'
                   '  renumberClustersContiguously(c, 4);\n'
                   '  buildNextLevelGraphOpt(g, o, c, 2, 1);\n'
                   '  vertexFollowing(g, c);\n'
                   '  buildNewGraphVF(g, o, c, 2);\n'
                   '  algoColoringMultiHashMaxMin(g, col, 1, t, 2, 4);\n'
                   '  removeEdges(4, 2, g->edgeList);\n'
                   '  SortEdgesUndirected(4, 2, g->edgeList, o->edgeList, c);\n'
                   '  SortNodeEdgesByIndex(4, g->edgeList, o->edgeList, c);\n'
                   '  parse_EdgeListBinaryNew(g, (char *)"f");\n'
                   '  writeGraphBinaryFormatNew(g, (char *)"f", 1);\n'
                   '  std::vector<long> v1, v2;\n'
                   '  computeCommunityComparisons(v1, 0, v2, 0);\n'
                   '  computeGiniCoefficient(c, 4);\n'
                   '  vBaseRedistribution(g, col, 4, 0);\n}\n')
    obj = tmp_path / 'use.o'
    subprocess.run(['g++', '-c', '-I', os.path.join(ROOT, 'include'), str(src), '-o', str(obj)],
                   check=True)
    undef = subprocess.run(['nm', '-u', str(obj)], capture_output=True, text=True).stdout
    for s in REFERENCE_SYMBOLS:
        assert s in undef


def test_no_gpu_fails_loudly():
    """Without a CUDA device the entry points return an error, never a CPU result."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    from grappolo_b200 import graphs, louvain
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.runMultiPhaseColoring(graphs.from_edges(2, [(0, 1)]))
    assert e.value.code == 7


def test_binary_files_through_the_library(tmp_path):
    """glv_load_binary / glv_write_binary (host file I/O, no GPU needed) read
    the reference-written karate.bin and write the same bytes back."""
    import numpy as np
    from grappolo_b200 import louvain
    path = os.path.join(ROOT, 'tests', 'golden', 'karate.bin')
    g, ne = louvain.parse_EdgeListBinaryNew(path)
    z = np.load(os.path.join(ROOT, 'tests', 'golden', 'karate.npz'))
    assert ne == 78
    assert np.array_equal(g.ptr, z['ptr']) and np.array_equal(g.tail, z['tail'])
    assert np.array_equal(g.weight, z['weight'])
    out = tmp_path / 'k.bin'
    louvain.writeGraphBinaryFormatNew(g, str(out))
    assert out.read_bytes() == open(path, 'rb').read()
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.parse_EdgeListBinaryNew(str(tmp_path / 'missing.bin'))
    assert e.value.code == 9  # GLV_ERR_IO
    (tmp_path / 'short.bin').write_bytes(open(path, 'rb').read()[:100])
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.parse_EdgeListBinaryNew(str(tmp_path / 'short.bin'))
    assert e.value.code == 9
