"""The C-ABI library loads and exports every entry point of include/sac_gpu.h (CPU).

No compute call is made here; on a machine without a GPU sac_create must fail
cleanly with SAC_ERR_NODEVICE instead of crashing or falling back to the CPU."""
import ctypes
import os
import re

import pytest

from sac_b200 import abi, build, params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "sac_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sac_[a-z_]+)\s*\(", text)))


def test_header_declares_the_reference_facing_calls():
    names = declared()
    for n in ("sac_create", "sac_set_grid", "sac_set_boundaries", "sac_upload", "sac_download",
              "sac_getboundary", "sac_getdt", "sac_advect", "sac_diag", "sac_last_error", "sac_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_oracle_exports_the_same_shape():
    from oracle import oracle

    lib = ctypes.CDLL(oracle.build())
    extensions = {"sac_default_params", "sac_synchronize", "sac_set_stream", "sac_get_stream", "sac_profile",
                  "sac_profile_read", "sac_kernel_launches", "sac_getdt_static"}
    for n in declared():
        if n in extensions or n.startswith("sac_batch_"):
            continue
        assert hasattr(lib, "oracle_" + n[4:]), n


def test_no_device_is_an_error_not_a_fallback():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = ctypes.CDLL(build.build())
    h = ctypes.c_void_p()
    p = params.default_params()
    assert lib.sac_create(ctypes.byref(p), ctypes.byref(h)) == 8  # SAC_ERR_NODEVICE
    with pytest.raises(abi.SacError):
        abi.Context(p)


def test_default_params_match_par_default():
    lib = ctypes.CDLL(build.build())
    p = params.SacParams()
    lib.sac_default_params(ctypes.byref(p))
    assert p.courantpar == 0.8 and p.dtpar == -1.0 and p.typeadvance == b"twostep" and p.sourceunsplit == 1
