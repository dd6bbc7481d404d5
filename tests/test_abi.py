"""CPU: the C-ABI library loads and exports every function include/*.h declares."""

import ctypes
import glob
import os
import re
import subprocess

import pytest

from diskann_b200 import _native
from diskann_b200.index import Knn, KnnSearchError, Status

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:int32_t|void|uint32_t|int64_t)\s+(dk_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_functions():
    names = _declared_functions()
    assert "dk_search" in names and "dk_index_create" in names
    assert set(names) == set(_native.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    for name in _declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for name in _declared_functions():
        assert name in exported, name


def test_abi_version():
    assert _native.load().dk_abi_version() == 1


@pytest.mark.parametrize("k,l,bw,status", [(0, 10, 1, Status.K_ZERO), (1, 0, 1, Status.L_ZERO),
                                           (11, 10, 1, Status.L_LESS_THAN_K),
                                           (10, 10, 0, Status.BEAM_WIDTH_ZERO), (10, 10, 1, Status.OK)])
def test_knn_validate_through_abi(k, l, bw, status):
    """dk_knn_validate is host-only: it needs no GPU."""
    lib = _native.load()
    assert lib.dk_knn_validate(k, l, bw) == status
    if status != Status.OK:
        code, msg = _native.last_error()
        assert code == status and msg


@pytest.mark.parametrize("k,l,bw,status", [(0, 10, None, Status.K_ZERO), (1, 0, None, Status.L_ZERO),
                                           (11, 10, None, Status.L_LESS_THAN_K),
                                           (10, 10, 0, Status.BEAM_WIDTH_ZERO)])
def test_knn_python_mirror(k, l, bw, status):
    with pytest.raises(KnnSearchError) as ei:
        Knn(k, l, bw)
    assert ei.value.status == status
    assert _native.load().dk_knn_validate(k, l, 1 if bw is None else bw) == status


def test_index_create_rejects_bad_descriptors_without_gpu():
    """Argument checks run before any CUDA call."""
    lib = _native.load()
    d = _native.IndexDesc()
    h = ctypes.c_void_p()
    assert lib.dk_index_create(None, 0, ctypes.byref(h)) == Status.INVALID_ARGUMENT
    d.dim = 0
    assert lib.dk_index_create(ctypes.byref(d), 0, ctypes.byref(h)) == Status.INVALID_ARGUMENT
    d.dim = 4
    d.num_frozen = 0
    assert lib.dk_index_create(ctypes.byref(d), 0, ctypes.byref(h)) == Status.INVALID_ARGUMENT
