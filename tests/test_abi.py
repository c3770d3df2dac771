"""C-ABI library: loads, exports every declared entry point, validates
arguments on the host (no GPU needed for any of this)."""
import ctypes
import os
import re

import pytest

from pyscfad_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "defined")))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    decl = _declared_functions()
    assert "triples_energy_vjp" in decl and "triples_energy" in decl
    assert "triples_lno_energy_vjp" in decl and "triples_lno_workspace_size" in decl
    for name in decl:
        assert hasattr(lib, name), name


def test_workspace_size_is_host_only_and_monotone():
    lib = _lib.load()
    a = lib.triples_workspace_size(0, 5, 19, 1, 0)
    b = lib.triples_workspace_size(0, 5, 19, 1, 1)
    c = lib.triples_workspace_size(0, 40, 360, 1, 1)
    assert 0 < a < b < c
    assert lib.triples_workspace_size(0, 0, 19, 1, 1) == 0       # nocc < 1
    assert lib.triples_workspace_size(7, 5, 19, 1, 1) == 0       # bad precision


def test_invalid_arguments_rejected_before_any_cuda_call():
    lib = _lib.load()
    null = None
    rc = lib.triples_energy(null, 0, 0, 19, 1, *([null] * 7), null, 0, null)
    assert rc == 1
    rc = lib.triples_energy(null, 9, 5, 19, 1, *([null] * 7), null, 0, null)
    assert rc == 1
    # workspace too small is reported as such
    rc = lib.triples_energy(null, 0, 5, 19, 1, *([ctypes.c_void_p(16)] * 7), ctypes.c_void_p(16), 8,
                            ctypes.c_void_p(16))
    assert rc == 2


def test_status_strings():
    lib = _lib.load()
    assert lib.triples_status_string(0) == b"ok"
    assert b"workspace" in lib.triples_status_string(2)
    with pytest.raises(_lib.TriplesError):
        _lib.check(1, "probe")


def test_lno_plan_limits():
    """The LNO path takes nocc <= 64 in every precision; larger problems are refused on the host."""
    lib = _lib.load()
    a = lib.triples_lno_workspace_size(0, 5, 19, 1, 0)
    b = lib.triples_lno_workspace_size(0, 5, 19, 1, 1)
    assert 0 < a < b
    assert b > lib.triples_workspace_size(0, 5, 19, 1, 1)        # whole-chunk work arrays
    assert lib.triples_lno_workspace_size(1, 5, 19, 1, 1) > 0    # mixed precision
    assert lib.triples_lno_workspace_size(0, 65, 19, 1, 1) == 0  # nocc > 64
    null = None
    rc = lib.triples_lno_energy(null, 0, 65, 19, 1, *([null] * 8), null, 0, null)
    assert rc == 4   # TRIPLES_ERR_UNSUPPORTED
    rc = lib.triples_lno_energy(null, 0, 5, 19, 1, *([ctypes.c_void_p(16)] * 8), ctypes.c_void_p(16), 8,
                                ctypes.c_void_p(16))
    assert rc == 2   # workspace too small
    rc = lib.triples_lno_energy(null, 0, 5, 19, 1, null, *([ctypes.c_void_p(16)] * 7), ctypes.c_void_p(16),
                                1 << 40, ctypes.c_void_p(16))
    assert rc == 1   # mat missing


def test_df_plan():
    """DF-factor entry points: workspace holds the packed ovvv (and its cotangent); naux >= 1."""
    lib = _lib.load()
    a = lib.triples_df_workspace_size(0, 5, 19, 60, 0)
    b = lib.triples_df_workspace_size(0, 5, 19, 60, 1)
    assert lib.triples_workspace_size(0, 5, 19, 1, 1) < b and 0 < a < b
    assert lib.triples_df_workspace_size(0, 5, 19, 0, 1) == 0    # naux < 1
    null = None
    rc = lib.triples_energy_df(null, 0, 5, 19, 60, *([null] * 8), null, 0, null)
    assert rc == 2   # workspace check comes first on null workspace
    rc = lib.triples_energy_df(null, 0, 5, 19, 60, *([null] * 8), ctypes.c_void_p(256), 1 << 40,
                               ctypes.c_void_p(16))
    assert rc == 1   # inputs missing


def test_lno_workspace_fits_one_b200_at_the_largest_fragments():
    """The projected epilogue's whole-chunk arrays grow as nocc^3 Tv^3: the
    plan halves the virtual block for large nocc so that the workspace stays
    well inside 180 GB, and energy-only calls keep two of the four arrays."""
    lib = _lib.load()
    for prec in (0, 1):
        for o, v in ((40, 360), (48, 200), (64, 400)):
            grad = lib.triples_lno_workspace_size(prec, o, v, 1, 1)
            energy = lib.triples_lno_workspace_size(prec, o, v, 1, 0)
            assert 0 < energy < grad < 150e9, (prec, o, v, grad)


def test_options_are_per_call_and_validated():
    """Block size, chunk slice and accumulation segment travel with the call
    (triples_options): no process-wide setter exists, a NULL options pointer
    means the defaults, and negative settings are refused."""
    lib = _lib.load()
    for gone in ("triples_set_block_size", "triples_set_chunk_range", "triples_set_accumulation_segment"):
        assert not hasattr(lib, gone), gone
    base = lib.triples_workspace_size(1, 20, 180, 1, 1)
    assert lib.triples_workspace_size_ex(1, 20, 180, 1, 1, None) == base
    assert lib.triples_workspace_size_ex(1, 20, 180, 1, 1, ctypes.byref(_lib.options())) == base
    small = lib.triples_workspace_size_ex(1, 20, 180, 1, 1, ctypes.byref(_lib.options(block_size=4)))
    assert 0 < small < base
    # the default plan is not changed by an earlier call with other options
    assert lib.triples_workspace_size(1, 20, 180, 1, 1) == base
    assert lib.triples_workspace_size_ex(1, 20, 180, 1, 1, ctypes.byref(_lib.options(block_size=-1))) == 0
    assert lib.triples_workspace_size_ex(1, 20, 180, 1, 1, ctypes.byref(_lib.options(chunk_range=(-1, 0)))) == 0
    assert lib.triples_lno_workspace_size_ex(1, 20, 180, 1, 1, ctypes.byref(_lib.options(block_size=4))) < \
        lib.triples_lno_workspace_size(1, 20, 180, 1, 1)
    # energy-only calls may pass NULL gradient pointers; missing inputs are still refused
    null = None
    rc = lib.triples_energy_vjp_ex(null, 0, 5, 19, 1, *([null] * 7), 1.0, 0, None, ctypes.c_void_p(256),
                                   1 << 30, ctypes.c_void_p(256), *([null] * 7))
    assert rc == 1


def _batch_problems(shapes):
    arr = (_lib.Problem * len(shapes))()
    for i, (o, v) in enumerate(shapes):
        arr[i].nocc, arr[i].nvir, arr[i].ovvv_packed = o, v, 1
    return arr


def test_batch_workspace_covers_every_problem_and_the_job_tables():
    lib = _lib.load()
    shapes = [(4, 20), (6, 27), (5, 33), (12, 80)]
    arr = _batch_problems(shapes)
    for prec in (0, 1, 2):
        total = lib.triples_batch_workspace_size(prec, len(shapes), arr)
        singles = sum(lib.triples_workspace_size(prec, o, v, 1, 1) for o, v in shapes)
        assert total >= singles
        if prec > 0:   # mixed modes add the job tables of the chunk steps
            assert total > singles
    assert lib.triples_batch_workspace_size(1, 0, arr) == 0                 # no problems
    bad = _batch_problems([(0, 20)])
    assert lib.triples_batch_workspace_size(1, 1, bad) == 0                 # nocc < 1
    assert lib.triples_batch_workspace_size(7, len(shapes), arr) == 0       # bad precision


def test_batch_create_rejects_bad_arguments_before_any_cuda_call():
    lib = _lib.load()
    arr = _batch_problems([(4, 20)])
    handle = ctypes.c_void_p()
    assert lib.triples_batch_create(1, 1, arr, 1.0, None, 0, ctypes.byref(handle)) == 2     # no workspace
    assert lib.triples_batch_create(1, 1, arr, 1.0, ctypes.c_void_p(256), 8, ctypes.byref(handle)) == 2  # too small
    assert lib.triples_batch_create(1, 1, arr, 1.0, ctypes.c_void_p(256), 1 << 40, None) == 1      # no handle slot
    assert handle.value is None
    assert lib.triples_batch_run(None, None) == 1
    lib.triples_batch_destroy(None)
