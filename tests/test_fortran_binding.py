"""The Fortran side of the C-ABI: include/sac_gpu_mod.f90 (ISO_C_BINDING) and the
host build that rewrites program vac's call sites (sac_b200/fortran).

No Fortran compiler exists on these machines, so the module is checked against
the C header as text: the bind(C) derived types must have the C structs' fields
in the same order with the same types, so that C's layout rules (which
ISO_C_BINDING prescribes for interoperable types) give the same offsets as
offsetof; and every bind(C) interface must match its C prototype in name,
parameter count and the by-value / by-reference kind of each parameter."""
import os
import re
import shutil
import subprocess

import pytest

from sac_b200.fortran import host_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MOD = os.path.join(ROOT, "include", "sac_gpu_mod.f90")
HDR = os.path.join(ROOT, "include", "sac_gpu.h")

SIZES = {"real(c_double)": (8, 8), "integer(c_int)": (4, 4), "character(kind=c_char)": (1, 1),
         "integer(c_size_t)": (8, 8)}


def _module_text():
    with open(MOD) as f:
        return f.read()


def _fortran_type(text, name):
    """[(component, fortran type, element count)] of `type, bind(C) :: name`."""
    m = re.search(rf"type, bind\(C\) :: {name}\n(.*?)\n\s*end type {name}", text, re.S)
    assert m, name
    out = []
    for line in m.group(1).splitlines():
        line = line.split("!")[0].strip()
        if not line:
            continue
        ftype, decl = [s.strip() for s in line.split("::")]
        for part in re.findall(r"(\w+)(?:\((\d+)\))?", decl):
            out.append((part[0], ftype, int(part[1]) if part[1] else 1))
    return out


def _c_layout(fields):
    """Offsets and size by C's rules: each field at the next multiple of its
    alignment, the struct padded to its largest alignment."""
    off, maxal, offs = 0, 1, {}
    for name, ftype, n in fields:
        size, al = SIZES[ftype]
        off = (off + al - 1) // al * al
        offs[name] = off
        off += size * n
        maxal = max(maxal, al)
    return offs, (off + maxal - 1) // maxal * maxal


def _c_offsets(tmp_path, ctype, names):
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("gcc not found")
    src = tmp_path / f"off_{ctype}.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "sac_gpu.h"\nint main(void) {\n'
                   + "".join(f'  printf("%zu\\n", offsetof({ctype}, {n}));\n' for n in names)
                   + f'  printf("%zu\\n", sizeof({ctype}));\n  return 0;\n}}\n')
    exe = tmp_path / f"off_{ctype}"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    return dict(zip(names, vals[:-1])), vals[-1]


@pytest.mark.parametrize("ctype", ["sac_params", "sac_diag_out"])
def test_bind_c_types_have_the_c_layout(tmp_path, ctype):
    fields = _fortran_type(_module_text(), ctype)
    offs, size = _c_layout(fields)
    c_offs, c_size = _c_offsets(tmp_path, ctype, [f[0] for f in fields])
    assert offs == c_offs
    assert size == c_size


def _c_prototypes():
    with open(HDR) as f:
        text = re.sub(r"/\*.*?\*/", " ", f.read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(sac_\w+)\s*\(([^;{]*?)\)\s*;", text):
        params = [p.strip() for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        protos[m.group(1)] = params
    return protos


def _fortran_interfaces(text):
    """{C name: [(argument, by value)]} of every bind(C) interface body."""
    out = {}
    for m in re.finditer(r"(?:function|subroutine)\s+(\w+)\(([^)]*)\)\s*&?\s*bind\(C, name='(\w+)'\)(.*?)"
                         r"end (?:function|subroutine)", text, re.S):
        args = [a.strip() for a in m.group(2).split(",") if a.strip()]
        body = m.group(4)
        byval = set()
        for line in body.splitlines():
            if "::" in line and "value" in line.split("::")[0]:
                byval.update(a.strip() for a in re.findall(r"(\w+)(?:\([^)]*\))?", line.split("::")[1]))
        out[m.group(3)] = [(a, a in byval) for a in args]
    return out


def test_interfaces_match_the_c_prototypes():
    protos = _c_prototypes()
    ifaces = _fortran_interfaces(_module_text())
    core = {"sac_default_params", "sac_create", "sac_set_grid", "sac_set_boundaries", "sac_upload", "sac_download",
            "sac_getboundary", "sac_getdt", "sac_getdt_static", "sac_advect", "sac_diag", "sac_synchronize",
            "sac_last_error", "sac_destroy"}
    assert core <= set(ifaces)
    for name, args in ifaces.items():
        if name == "strlen":
            continue
        assert name in protos, name
        params = protos[name]
        assert len(params) == len(args), (name, params, args)
        for (arg, byval), cparam in zip(args, params):
            pointer = "*" in cparam or "[" in cparam
            # by value: a C scalar, or a pointer passed as type(c_ptr), value
            if byval:
                assert not pointer or arg in ("ctx", "c", "s") or cparam.startswith(("sac_ctx", "const sac_ctx")), \
                    (name, arg, cparam)
            else:
                assert pointer, (name, arg, cparam)


def _synthetic_vac():
    """A stand-in for src/vac.t that holds each pattern the host build rewrites."""
    lines = ["program vac", "call startup", "call getboundary(t,1,nw,1,ndim,w)", "do",
             "   do ifile=1,nfile", "      if(timetosave(ifile)) call savefile(ifile,w)", "   end do",
             "   " + host_build.DT_BLOCK_START]
    lines += ["      " + s for s in host_build.DT_BLOCK_LINES]
    lines += ["   if(dtmrpc>zero)dt=min(dt,dtmrpc)",
              "   if(residmin>zero .or. residmax<bigdouble)then\n      ! calculate true residual", "   endif",
              "end do", "   if(itsavelast(ifile)<it)call savefile(ifile,w)",
              "if(verbose)write(*,'(a,f10.3,a)')'Finish Advance ',time1,' sec'", "end",
              "subroutine advance_expl(method,ix^L,iws,w1,w)",
              "         call advect(method,ix^L,iws,idimsplit,idimsplit,w1,w)",
              "         call advect(method,ix^L,iws,idimsplit,idimsplit,w1,w)",
              "   call advect(method,ix^L,iws,1,ndim,w1,w)", "end"]
    return "\n".join(lines) + "\n"


def test_call_sites_are_rewritten():
    out = host_build.patch_vac(_synthetic_vac())
    assert "call gpuini(w)" in out and "call gpugetdt(w)" in out and "call gpufinish" in out
    assert out.count("call gpuadvect(") == 3 and out.count("call gpudownload(w)") == 3
    for gone in ("getdt_courant", "call advect(", "call getboundary(", "dt=dtpar"):
        assert gone not in out, gone
    assert "if(dtmrpc>zero)dt=min(dt,dtmrpc)" in out  # stays on the host


def test_a_changed_reference_is_refused():
    text = _synthetic_vac().replace("call getdt(w,ixM^L)", "call getdt(w,ixM^L,1)")
    with pytest.raises(host_build.PatchError):
        host_build.patch_vac(text)
    text = _synthetic_vac().replace("   call advect(method,ix^L,iws,1,ndim,w1,w)\n", "")
    with pytest.raises(host_build.PatchError):
        host_build.patch_vac(text)


@pytest.mark.skipif(not os.environ.get("SAC_REFERENCE"), reason="SAC_REFERENCE (the SAC tree) not set")
def test_the_reference_main_program_patches():
    with open(os.path.join(os.environ["SAC_REFERENCE"], "src", "vac.t")) as f:
        out = host_build.patch_vac(f.read())
    assert "call gpugetdt(w)" in out


def test_shim_calls_only_declared_entry_points():
    with open(host_build.SHIM) as f:
        shim = f.read()
    declared = set(_fortran_interfaces(_module_text())) | {"sac_error_text", "sac_set_name"}
    called = set(re.findall(r"\b(sac_\w+)\s*\(", shim))
    assert called <= declared, called - declared


def test_host_build_needs_a_fortran_compiler(tmp_path):
    if host_build.fortran_compiler() is not None:
        pytest.skip("a Fortran compiler is present")
    with pytest.raises(RuntimeError, match="no Fortran compiler"):
        host_build.build(str(tmp_path), str(tmp_path / "out"))
