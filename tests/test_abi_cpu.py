"""C-ABI library checks that need no GPU: it loads, exports every symbol the
header declares, and its host-side parameter logic matches the Python mirror."""
import ctypes as C
import os
import re

import pytest

from gpg.abi import GPG_MG, GPG_SOR, GpgParams, default_params
from gpg.lib import GpgError, LIB_PATH, check, library

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in os.listdir(os.path.join(REPO, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(REPO, "include", h)).read()
            names += re.findall(r"^GPG_API\s+[^;(]*?\b(gpg_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB_PATH), "build with gpu_testbed_poisson-gravity_b200/build.py"
    lib = C.CDLL(LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n


def test_params_struct_layout_matches_header():
    # field offsets of struct gpg_params (include/gpg.h), naturally aligned
    # (sizeof/offsetof as compiled by gcc from include/gpg.h)
    assert C.sizeof(GpgParams) == 112
    assert GpgParams.dt.offset == 32 and GpgParams.mg_tolerated_error.offset == 80
    assert GpgParams.sor_tolerance.offset == 104


@pytest.mark.parametrize("rs", [4, 8])
@pytest.mark.parametrize("g", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("scheme", [GPG_SOR, GPG_MG])
def test_c_defaults_equal_python_defaults(rs, g, scheme):
    p = GpgParams()
    check(library().gpg_default_params(C.byref(p), rs, g, scheme))
    assert p.as_dict() == default_params(rs, g, scheme).as_dict()
    check(library().gpg_validate_params(C.byref(p)))


@pytest.mark.parametrize("field,value", [("ghost", 0), ("ghost", 6), ("gra_ghost", 3), ("int_scheme", 1),
                                         ("real_size", 2), ("scheme", 3), ("init_mode", 7),
                                         ("stop_mode", 4), ("sor_max_iter", -1), ("p5_gradient", 1)])
def test_validation_rejects(field, value):
    p = default_params(4, 1, GPG_SOR).copy(**{field: value})
    rc = library().gpg_validate_params(C.byref(p))
    assert rc == 1
    assert library().gpg_last_error()


def test_patch_sizes():
    p = default_params(4, 5, GPG_SOR, gra_ghost=2)
    v = [C.c_int64() for _ in range(4)]
    check(library().gpg_patch_sizes(C.byref(p), *[C.byref(x) for x in v]))
    assert [x.value for x in v] == [16 ** 3, 12 ** 3, 12 ** 3, 2560]


def test_device_call_without_gpu_reports_error():
    """Without a CUDA device the library returns an error status, never a CPU result."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(GpgError):
        from gpg.lib import set_diagnose_device
        set_diagnose_device(0)


def test_sor_variant_table_queries():
    """The variant table answers without a GPU: 17 launch shapes, each with a
    CTA size (0: staged persistent), pass order and layout; out-of-range ids
    are rejected."""
    lib = library()
    n = lib.gpg_sor_variant_count()
    assert n == 17
    shapes = set()
    for v in range(n):
        ppc, ph, z, y, st = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib.gpg_sor_variant_info(v, C.byref(ppc), C.byref(ph)))
        check(lib.gpg_sor_variant_layout(v, C.byref(z), C.byref(y)))
        check(lib.gpg_sor_variant_staged(v, C.byref(st)))
        assert ph.value in (0, 1) and z.value in (1, 2) and y.value in (1, 2)
        assert (ppc.value == 0) == bool(st.value) and ppc.value in (0, 1, 2, 4)
        shapes.add((ppc.value, ph.value, z.value, y.value))
    assert len(shapes) == n  # no two variants alike
    for bad in (-1, n):
        with pytest.raises(GpgError):
            check(lib.gpg_sor_variant_layout(bad, None, None))
    with pytest.raises(GpgError):
        check(lib.gpg_set_sor_variant(4, 3, n))
    with pytest.raises(GpgError):
        check(lib.gpg_set_sor_variant(4, 3, -2))
    # -1 hands the choice back to the library: its built-in large-batch variant
    before = C.c_int()
    check(lib.gpg_get_sor_variant(4, 3, C.byref(before)))
    check(lib.gpg_set_sor_variant(4, 3, (before.value + 1) % n))
    check(lib.gpg_set_sor_variant(4, 3, -1))
    after = C.c_int()
    check(lib.gpg_get_sor_variant(4, 3, C.byref(after)))
    assert after.value == before.value


def test_launch_size_choice_of_sor_variants():
    """Small launches take their own built-in variant until one is set; a set
    variant holds at every size; -1 restores the library's choice."""
    lib = library()
    n = lib.gpg_sor_variant_count()
    v = C.c_int()

    def at(npatch):
        check(lib.gpg_sor_variant_for_launch(4, 1, npatch, C.byref(v)))
        return v.value

    large = C.c_int()
    check(lib.gpg_get_sor_variant(4, 1, C.byref(large)))
    small = at(64)
    assert at(1 << 20) == large.value and small != large.value
    assert at(2048) == small and at(2049) == large.value
    check(lib.gpg_set_sor_variant(4, 1, (large.value + 1) % n))
    try:
        assert at(64) == at(1 << 20) == (large.value + 1) % n
    finally:
        check(lib.gpg_set_sor_variant(4, 1, -1))
    assert at(64) == small and at(1 << 20) == large.value
    with pytest.raises(GpgError):
        check(lib.gpg_sor_variant_for_launch(4, 1, -1, C.byref(v)))
