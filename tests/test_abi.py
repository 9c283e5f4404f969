"""The C-ABI library: it loads, exports what include/thunderstep.h declares, and its
built-in kernel table is the reference's kernel ABI.  No compute calls here."""
import ctypes
import json
import os
import re

import pytest

from tests import helpers

ROOT = helpers.ROOT
HEADER = os.path.join(ROOT, 'include', 'thunderstep.h')


def _declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r'\b(te_[a-z_0-9]+)\s*\(', src)))


def _lib():
    from thunderengine_web_b200 import replayer
    return replayer.load_library()


def test_library_exports_every_declared_symbol():
    lib = _lib()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_python_bindings_cover_the_header():
    from thunderengine_web_b200 import replayer
    assert set(_declared()) <= set(replayer.EXPORTS)


def test_kernel_table_is_the_reference_abi():
    lib = _lib()
    n = lib.te_kernel_table_json(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib.te_kernel_table_json(buf, n + 1)
    table = json.loads(buf.value.decode())
    ref = helpers.kernels_meta()
    assert len(table) == 84
    for name, k in table.items():
        want = [(p['index'], p['kind'], bool(p['write'])) for p in ref[name]['params']]
        got = [(p['index'], p['kind'], bool(p['write'])) for p in k['params']]
        assert got == want, name
        # per-thread scratch: only the Morrison column and its reflectivity diagnostic have
        # some (their per-column arrays)
        assert ref[name]['scratch'] == {'morr_column': 3712, 'morr_refl10cm': 1408}.get(name, 0), name


def test_oracle_declares_the_same_kernels():
    lib = _lib()
    n = lib.te_kernel_table_json(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib.te_kernel_table_json(buf, n + 1)
    table = json.loads(buf.value.decode())
    o = helpers.oracle()
    for name in table:
        if name in ('morr_column', 'morr_refl10cm'):
            # checked against the reference's own kernels (tests/test_morr.py)
            continue
        assert o.has(name), name


def test_region_hash_host_matches_reference_formula():
    from oracle.player import region_hash
    import numpy as np
    lib = _lib()
    w = np.arange(1000, dtype=np.uint32) * np.uint32(2654435761)
    assert lib.te_region_hash_host(w.ctypes.data_as(ctypes.c_void_p), w.size) == region_hash(w)


def test_errors_are_reported_not_raised_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip('checks the no-GPU error path')
    from thunderengine_web_b200.replayer import Replayer
    with pytest.raises(RuntimeError):
        Replayer({'buffers': []})
