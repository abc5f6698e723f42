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
    # the C defaults and the Python mirror's agree field by field
    q = params.default_params()
    for name, ctype in params.SacParams._fields_:
        a, b = getattr(p, name), getattr(q, name)
        if isinstance(a, (bytes, int, float)):
            assert a == b, name
        else:
            assert list(a) == list(b), name


C_CALLER = r"""
#include <stdio.h>
#include <string.h>
#include "sac_gpu.h"
#include "sac_fno.h"

int main(void) {
  sac_params p;
  sac_ctx* c = NULL;
  sac_status st;
  sac_default_params(&p);
  strcpy(p.typeadvance, "fourstep");
  st = sac_create(&p, &c);
  printf("%d %zu %d %s %.17g %d\n", (int)st, sizeof(sac_params), p.sourceunsplit, p.typeadvance, p.courantpar,
         c == NULL);
  if (c) sac_destroy(c);
  return 0;
}
"""


def test_headers_compile_as_c99_and_a_c_caller_links(tmp_path):
    """A C host (the Fortran shim's ISO_C_BINDING side sees the same layout)
    includes both headers with a strict C99 compiler, links the library and
    calls it; without a GPU sac_create returns SAC_ERR_NODEVICE and no context."""
    import shutil
    import subprocess

    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("gcc not found")
    path = build.build()
    src = tmp_path / "caller.c"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), path, "-Wl,-rpath," + os.path.dirname(path)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    status = params.STATUS[int(out[0])]
    assert status in ("SAC_OK", "SAC_ERR_NODEVICE")
    assert out[5] == ("1" if status == "SAC_ERR_NODEVICE" else "0")
    assert int(out[1]) == ctypes.sizeof(params.SacParams)
    assert out[2] == "1" and out[3] == "fourstep" and float(out[4]) == 0.8


def _c_offsets(tmp_path, header, ctype, names):
    import shutil
    import subprocess

    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("gcc not found")
    src = tmp_path / f"offsets_{ctype}.c"
    src.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "{header}"\nint main(void) {{\n'
                   + "".join(f'  printf("%zu\\n", offsetof({ctype}, {n}));\n' for n in names)
                   + f'  printf("%zu\\n", sizeof({ctype}));\n  return 0;\n}}\n')
    exe = tmp_path / f"offsets_{ctype}"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    return [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]


@pytest.mark.parametrize("header,ctype,mirror", [("sac_gpu.h", "sac_params", "sac_b200.params:SacParams"),
                                                 ("sac_gpu.h", "sac_diag_out", "sac_b200.params:SacDiag"),
                                                 ("sac_fno.h", "sac_fno_gemm_desc", "sac_b200.fno_abi:GemmDesc"),
                                                 ("sac_fno.h", "sac_fno_config", "sac_b200.fno_abi:FnoConfig")])
def test_struct_layouts_match_the_c_headers(tmp_path, header, ctype, mirror):
    """Every field of the ctypes mirrors sits at the offset the C compiler gives
    the same field of the header's struct, and the sizes agree."""
    import importlib

    mod, cls = mirror.split(":")
    S = getattr(importlib.import_module(mod), cls)
    names = [f[0] for f in S._fields_]
    got = _c_offsets(tmp_path, header, ctype, names)
    want = [getattr(S, n).offset for n in names] + [ctypes.sizeof(S)]
    assert got == want, list(zip(names + ["sizeof"], got, want))
