"""CPU checks of the C ABI: the library loads, exports every entry point the
header declares, and rejects bad configurations with fosite's error classes
before touching a device."""
import ctypes as C
import os
import re

import pytest

from fosite_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fosite_gpu.h")


def _declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|int64_t)\s+(fgpu_\w+)\s*\(", txt, flags=re.M)))


@pytest.mark.parametrize("exact", [False, True])
def test_library_exports_header_symbols(exact):
    from fosite_b200.sim import lib_path
    path = lib_path(exact)
    if not os.path.exists(path):
        pytest.skip("library not built")
    L = C.CDLL(path)
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def _create(cfg):
    from fosite_b200.sim import lib
    L = lib()
    h = C.c_void_p()
    rc = L.fgpu_create(C.byref(cfg), -1, C.byref(h))
    buf = C.create_string_buffer(256)
    L.fgpu_last_error(None, buf, 256)
    if rc == 0:
        L.fgpu_destroy(h)
    return rc, buf.value.decode()


def _cfg(**kw):
    c = abi.default_config()
    c.inum, c.jnum, c.knum = 16, 16, 1
    c.xmin, c.xmax, c.ymin, c.ymax = 0.0, 1.0, 0.0, 1.0
    c.tol_rel = 10.0
    for k, v in kw.items():
        setattr(c, k, v)
    return abi.finalize_config(c)


@pytest.mark.parametrize("kw,code", [
    (dict(limiter=abi.PP), abi.EUNSUPPORTED),
    (dict(limiter=42), abi.EBADCFG),
    (dict(physics=3), abi.EBADCFG),
    (dict(geometry=40), abi.EUNSUPPORTED),
    (dict(method=9), abi.EBADCFG),
    (dict(jnum=1), abi.EUNSUPPORTED),
    (dict(fluxtype=2), abi.EBADCFG),
    # FARGO: types 1 and 2 along x or y on 2D meshes
    (dict(physics=abi.EULER_ISOTHERM, csiso=1.0, fargo_method=3, fargo_direction=2), abi.EUNSUPPORTED),
    (dict(physics=abi.EULER_ISOTHERM, csiso=1.0, fargo_method=1, fargo_direction=3), abi.EUNSUPPORTED),
    (dict(physics=abi.EULER_ISOTHERM, csiso=1.0, fargo_method=1, fargo_direction=1, pointmass=1, pm_outbound=1,
          geometry=abi.CYLINDRICAL, xmin=0.5, xmax=1.5), abi.EUNSUPPORTED),
    (dict(fargo_method=1, fargo_direction=2), abi.EUNSUPPORTED),
])
def test_bad_configs_rejected(kw, code):
    from fosite_b200.sim import lib_path
    if not os.path.exists(lib_path()):
        pytest.skip("library not built")
    rc, msg = _create(_cfg(**kw))
    assert rc == code, (rc, msg)
    assert msg


def test_unpaired_periodic_rejected():
    from fosite_b200.sim import lib_path
    if not os.path.exists(lib_path()):
        pytest.skip("library not built")
    c = _cfg()
    c.bc[abi.WEST] = abi.REFLECTING
    rc, msg = _create(c)
    assert rc == abi.EBADCFG and "periodic" in msg


def test_struct_layout_matches_header():
    # offsets of the ctypes mirror must match the C compiler's (checked with a tiny C program)
    import subprocess
    import tempfile
    fields = [f[0] for f in abi.Config._fields_]
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"%s\"\nint main(){\n" % HEADER
    for f in fields:
        src += 'printf("%%zu\\n", offsetof(fgpu_config, %s));\n' % f
    src += 'printf("%zu\\n", sizeof(fgpu_config)); printf("%zu\\n", sizeof(fgpu_status)); printf("%zu\\n", sizeof(fgpu_stats)); return 0;}\n'
    with tempfile.TemporaryDirectory() as d:
        cpath = os.path.join(d, "t.c")
        open(cpath, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.check_call(["gcc", "-o", exe, cpath])
        out = [int(x) for x in subprocess.check_output([exe]).split()]
    for f, off in zip(fields, out):
        assert getattr(abi.Config, f).offset == off, f
    assert out[len(fields)] == C.sizeof(abi.Config)
    assert out[len(fields) + 1] == C.sizeof(abi.Status)
    assert out[len(fields) + 2] == C.sizeof(abi.Stats)
