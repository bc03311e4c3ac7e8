"""The C ABI library loads on a machine without a GPU, exports every entry point include/cdd.h
declares, and its struct layout matches the ctypes binding (checked against gcc)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "cdd.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cdd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from cdd import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.exported_names())
    assert lib.cdd_version().decode().startswith("cdd-b200")
    assert lib.cdd_last_error() is not None


def test_instance_struct_layout_matches_ctypes(tmp_path):
    from cdd import _lib
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "%s"\n'
                   'int main(void){printf("%%zu %%zu %%zu %%zu %%zu %%zu %%zu %%zu %%zu %%zu\\n", sizeof(cdd_instance),'
                   'offsetof(cdd_instance, mu), offsetof(cdd_instance, has_load),'
                   'offsetof(cdd_instance, load_rate), offsetof(cdd_instance, load_t0),'
                   'offsetof(cdd_instance, load_nu), offsetof(cdd_instance, dynamics),'
                   'offsetof(cdd_instance, vacancy), offsetof(cdd_instance, vac_gamma),'
                   'offsetof(cdd_instance, dt_max)); return 0;}\n' % HEADER)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    S = _lib.cdd_instance
    assert got == [ctypes.sizeof(S), S.mu.offset, S.has_load.offset, S.load_rate.offset,
                   S.load_t0.offset, S.load_nu.offset, S.dynamics.offset, S.vacancy.offset,
                   S.vac_gamma.offset, S.dt_max.offset]


def test_noalloc_rejects_oversize_grid_without_touching_the_gpu():
    from cdd import _lib
    lib = _lib.load()
    inst = _lib.cdd_instance()
    inst.ndim = 3
    inst.shape[0] = inst.shape[1] = inst.shape[2] = 256
    inst.mu, inst.nu = 1.0, 0.3
    rc = lib.cdd_stress_noalloc(ctypes.byref(inst), _lib.CDD_F64, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                ctypes.c_void_p(0))
    assert rc == _lib.CDD_ERR_SHAPE
    assert "scratch" in lib.cdd_last_error().decode()


def test_plan_create_rejects_bad_shapes_before_device_work():
    from cdd import _lib
    lib = _lib.load()
    for shape, nd in [((7, 8, 8), 3), ((14, 8, 8), 3), ((8, 8, 2048), 3), ((8, 8, 0), 2)]:
        inst = _lib.cdd_instance()
        inst.ndim = nd
        for a in range(3):
            inst.shape[a] = shape[a]
        inst.mu, inst.nu, inst.cfl = 1.0, 0.3, 0.25
        h = ctypes.c_void_p()
        rc = lib.cdd_plan_create(ctypes.byref(inst), 1, _lib.CDD_F64, ctypes.byref(h))
        if nd == 2 and shape[1] == 8:
            continue
        assert rc == _lib.CDD_ERR_SHAPE, shape
        assert not h.value


def test_tuning_struct_layout_matches_ctypes(tmp_path):
    from cdd import _lib
    src = tmp_path / "tlayout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "%s"\n'
                   'int main(void){printf("%%zu %%zu %%zu %%zu\\n", sizeof(cdd_tuning),'
                   'offsetof(cdd_tuning, green_cols), offsetof(cdd_tuning, stencil_planes),'
                   'offsetof(cdd_tuning, plane_fft)); return 0;}\n' % HEADER)
    exe = tmp_path / "tlayout"
    subprocess.run(["gcc", "-std=c99", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    S = _lib.cdd_tuning
    assert got == [ctypes.sizeof(S), S.green_cols.offset, S.stencil_planes.offset, S.plane_fft.offset]


def test_tuned_plan_rejects_bad_tuning_before_device_work():
    from cdd import _lib
    lib = _lib.load()
    inst = _lib.cdd_instance()
    inst.ndim = 3
    for a in range(3):
        inst.shape[a] = 16
    inst.mu, inst.nu, inst.cfl = 1.0, 0.3, 0.25
    for bad in [dict(fft_radix=32), dict(fft_radix=2), dict(mid_cols=12), dict(green_cols=128),
                dict(rows_lines=5000), dict(stencil_planes=-1), dict(plane_fft=2), dict(plane_fft=-2)]:
        t = _lib.cdd_tuning.from_dict(bad)
        h = ctypes.c_void_p()
        rc = lib.cdd_plan_create_tuned(ctypes.byref(inst), 1, _lib.CDD_F64, ctypes.byref(t), ctypes.byref(h))
        assert rc == _lib.CDD_ERR_ARG, bad
        assert "tuning" in lib.cdd_last_error().decode()


def test_documented_binding_struct_matches_header(tmp_path):
    """The ctypes cdd_instance a maintainer copies from INTEGRATION.md section 2 has every field of
    include/cdd.h at gcc's offsets, and the same size, so the library never reads past its end."""
    text = open(os.path.join(REPO, "INTEGRATION.md")).read()
    block = re.search(r"^class cdd_instance\(ctypes\.Structure\):.*?\]\n", text, flags=re.M | re.S)
    assert block, "INTEGRATION.md has no ctypes cdd_instance"
    ns = {"ctypes": ctypes}
    exec(block.group(0), ns)
    S = ns["cdd_instance"]
    names = [f[0] for f in S._fields_]
    hdr = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct cdd_instance \{(.*?)\} cdd_instance;", hdr, flags=re.S).group(1)
    declared = re.findall(r"(\w+)(?:\[\d+\])?\s*[,;]", body)
    assert names == declared
    src = tmp_path / "doc_layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "%s"\nint main(void){\n'
                   'printf("%%zu\\n", sizeof(cdd_instance));\n%s return 0;}\n'
                   % (HEADER, "".join('printf("%%zu\\n", offsetof(cdd_instance, %s));\n' % n for n in names)))
    exe = tmp_path / "doc_layout"
    subprocess.run(["gcc", "-std=c99", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert got == [ctypes.sizeof(S)] + [getattr(S, n).offset for n in names]
