"""CPU tests of the boundary: the C-ABI library loads and exports every entry
point include/gbgpu.h declares, the mirrored structs have the reference's
byte layout, and the host-side containers/generators keep the contract.
No compute call is made here (there is no GPU on the CPU runner)."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from gb_b200 import _lib, la, synth
from gb_b200.matrix import MacaulayMatrix, ff_bits, kernel_family

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "gbgpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    names = re.findall(r"\b(gbgpu_[a-z_0-9]+)\s*\(", src)
    return sorted(set(names))


def test_header_lists_match_binding():
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    for name in declared_functions():
        assert name in exported, name
        assert getattr(lib, name) is not None


def test_library_is_sm100a_only():
    out = subprocess.run(["cuobjdump", "--list-elf", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    assert "sm_100a" in out


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_mirrored_struct_layout_matches_reference():
    want = oracle.ref_layout()
    got = la.layout()
    assert got.tolist() == want.tolist()


def test_ff_bits_and_family_follow_reference_dispatch():
    assert [ff_bits(p) for p in (2, 101, 127, 128, 251, 32003, 32768, 65521, 2147483647)] == \
        [8, 8, 8, 16, 16, 16, 32, 32, 32]
    assert kernel_family(65521) == "17_bit" and kernel_family(131071) == "17_bit" \
        and kernel_family(2147483647) == "31_bit"


def test_staircase_generator_contract():
    m = synth.staircase(300, 80, 300, 65521, seed=2)
    m.validate()
    nru, nrl = m.split_counts()
    assert (nru, nrl) == (300, 80)
    lens = np.diff(m.row_ptr)
    dens = lens / m.nc
    assert dens.min() >= 0.015 and dens.max() <= 0.055
    # deterministic
    m2 = synth.staircase(300, 80, 300, 65521, seed=2)
    assert np.array_equal(m.cols, m2.cols) and np.array_equal(m.vals, m2.vals)


def test_validate_catches_contract_violations():
    m = synth.random_macaulay(10, 6, 12, 101, seed=4)
    m.validate()
    bad = MacaulayMatrix(m.p, m.ncl, m.ncr, m.row_ptr, m.cols.copy(), m.vals)
    bad.cols[-1] = m.nc  # column out of range
    with pytest.raises(ValueError):
        bad.validate()
    bad = MacaulayMatrix(m.p, m.ncl, m.ncr, m.row_ptr, m.cols, m.vals.copy())
    bad.vals[-1] = m.p  # coefficient out of range
    with pytest.raises(ValueError):
        bad.validate()


def test_dense_lowrank_rank():
    D = synth.dense_lowrank(12, 15, 5, 101, seed=1)
    # rank over GF(101) by plain elimination
    A = D.copy() % 101
    r = 0
    for c in range(A.shape[1]):
        piv = next((i for i in range(r, A.shape[0]) if A[i, c] % 101), None)
        if piv is None:
            continue
        A[[r, piv]] = A[[piv, r]]
        inv = pow(int(A[r, c]), 99, 101)
        A[r] = (A[r] * inv) % 101
        for i in range(A.shape[0]):
            if i != r and A[i, c]:
                A[i] = (A[i] - A[i, c] * A[r]) % 101
        r += 1
    assert r == 5


@pytest.mark.skipif(not oracle.gb_gpu_available(), reason="integration build absent")
def test_integration_recipe_build_links_to_library():
    """The two-macro drop-in recipe reroutes only the two call sites: the gb build
    exports f4_julia and imports exactly the two GPU entry points."""
    out = subprocess.run(["nm", "-D", oracle.GB_GPU_SO], capture_output=True, text=True,
                         check=True).stdout
    undefined = set(re.findall(r" U (gbgpu_\w+)", out))
    assert undefined == {"gbgpu_linear_algebra", "gbgpu_interreduce_matrix_rows"}
    assert re.search(r" T f4_julia\b", out)


def test_steps_around_the_la_reject_bad_calls_before_any_device_work():
    """The basis conversion needs the kept answer of gbgpu_linear_algebra_keep
    for the same matrix, and symbolic preprocessing tables over the same
    variables with a power-of-two map: both refuse otherwise, with
    GBGPU_EINVAL, before touching the device."""
    import ctypes as C
    lib = _lib.load()
    mat = (C.c_uint8 * 256)()
    bs = (C.c_uint8 * 256)()
    st = (C.c_uint8 * 1024)()
    bht = (C.c_int32 * 32)()
    sht = (C.c_int32 * 32)()
    hcm = (C.c_int32 * 4)()
    lib.gbgpu_kept_answer.argtypes = [C.c_void_p]
    assert lib.gbgpu_kept_answer(C.addressof(mat)) == 0
    f = lib.gbgpu_convert_sparse_matrix_rows_to_basis_elements_status
    f.argtypes = [C.c_void_p] * 6
    assert f(C.addressof(mat), C.addressof(bs), C.addressof(bht), C.addressof(sht),
             C.addressof(hcm), C.addressof(st)) == -22
    # ht_t: 3 pointers (6 int32 slots), then eld, esz, hsz, nv
    sht[6:10] = [1, 8, 16, 3]
    bht[6:10] = [1, 8, 16, 4]
    g = lib.gbgpu_symbolic_preprocessing_status
    g.argtypes = [C.c_void_p] * 5
    assert g(C.addressof(mat), C.addressof(bs), C.addressof(st), C.addressof(sht),
             C.addressof(bht)) == -22
    bht[9] = 3
    sht[8] = 12  # not a power of two
    assert g(C.addressof(mat), C.addressof(bs), C.addressof(st), C.addressof(sht),
             C.addressof(bht)) == -22
