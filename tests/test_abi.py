"""The C-ABI library loads and exports every symbol include/pofd_b200.h
declares; host-side error paths behave like the reference's exceptions.
No GPU needed."""
import ctypes as C

import numpy as np
import pytest


def test_every_declared_symbol_is_exported(built_lib):
    from pofd_affine_b200 import _lib
    raw = C.CDLL(built_lib)
    decl = _lib.declared_functions()
    assert len(decl) >= 20
    missing = [n for n in decl if not hasattr(raw, n)]
    assert not missing, missing
    # and the Python binding covers all of them
    assert set(decl) <= set(_lib.SIGNATURES), set(decl) - set(_lib.SIGNATURES)


def test_support_library_exports_its_header(built_lib):
    """The measurement and test helpers live in libpofd_b200_support.so,
    declared in include/pofd_b200_support.h, and none of them in the
    likelihood's ABI."""
    from pofd_affine_b200 import _lib
    raw = C.CDLL(_lib.SUPPORT_LIBPATH)
    decl = _lib.declared_functions(_lib.SUPPORT_HEADER)
    assert set(decl) == set(_lib.SUPPORT_SIGNATURES)
    missing = [n for n in decl if not hasattr(raw, n)]
    assert not missing, missing
    main = C.CDLL(built_lib)
    assert not [n for n in decl if hasattr(main, n)]
    assert not set(decl) & set(_lib.declared_functions())


def test_version_and_no_error(built_lib):
    from pofd_affine_b200._lib import lib
    assert b"pofd_affine 0.5.1" in lib().pofd_version()


def test_zero_beam_raises_like_reference(host_ctx):
    from pofd_affine_b200 import PofdError, beam
    with pytest.raises(PofdError) as e:
        beam(np.zeros((5, 5)), 6.0)
    assert e.value.code == -10
    assert "only zero values" in str(e.value)


def test_bad_pixsize_and_knots(host_ctx):
    from pofd_affine_b200 import PofdError, beam, calcLike
    with pytest.raises(PofdError):
        beam(np.ones((5, 5)), 0.0)
    with pytest.raises(PofdError):
        calcLike(host_ctx, [0.01, 0.005, 0.02], 1024)  # not increasing
    with pytest.raises(PofdError):
        calcLike(host_ctx, [0.01, 0.02], 1024)  # fewer than 3 knots


def test_gpu_calls_fail_loudly_on_host_only_context(host_ctx):
    from pofd_affine_b200 import PofdError, beam, calcLike, synth
    L = calcLike(host_ctx, [0.002, 0.01, 0.05, 0.2], 1024, 64, True, 50)
    b = beam(synth.gaussian_beam(3.0), 6.0, True, 50)
    L.addBeamSet(b)
    L.addDataset(0, np.random.default_rng(0).normal(0, 0.002, 500), 0.002)
    L.setRRanges(np.array([5, 4, 3, 2, 1], np.float32))
    with pytest.raises(PofdError) as e:
        L.getLogLike(np.array([5, 4, 3, 2, 1], np.float32))
    assert e.value.code == -11


def test_setrranges_needs_valid_model(host_ctx):
    from pofd_affine_b200 import PofdError, beam, calcLike, synth
    L = calcLike(host_ctx, [0.002, 0.01, 0.05], 1024, 64, True, 50)
    L.addBeamSet(beam(synth.gaussian_beam(3.0), 6.0, True, 50))
    L.addDataset(0, np.linspace(-0.01, 0.01, 100), 0.002)
    with pytest.raises(PofdError) as e:
        L.setRRanges(np.array([5, np.nan, 3, 1], np.float32))
    assert e.value.code == -1
