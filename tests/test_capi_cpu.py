"""The C-ABI library builds, loads and exports every declared entry point
(no GPU needed: nothing is computed here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "gtb200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gtb_[a-z_0-9]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from gtalign_alpha_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def test_library_exports_every_declared_symbol(lib):
    names = declared()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n


def test_errors_without_device_are_status_codes(lib):
    """On a machine without a usable device the create call fails cleanly with
    GTB_ERR_CUDA (and never raises or aborts)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    from gtalign_alpha_b200.api import _COptions
    h = ctypes.c_void_p()
    opts = _COptions(1, 2, 18, 0.4, 0, 0, 0, 1, 0, 0)
    lib.gtb_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(_COptions),
                               ctypes.POINTER(ctypes.c_void_p)]
    st = lib.gtb_create(0, 0, ctypes.byref(opts), ctypes.byref(h))
    assert st == 2
    lib.gtb_last_error.restype = ctypes.c_char_p
    lib.gtb_last_error.argtypes = [ctypes.c_void_p]
    assert lib.gtb_last_error(h)
    lib.gtb_destroy.argtypes = [ctypes.c_void_p]
    lib.gtb_destroy(h)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from gtalign_alpha_b200 import api
    monkeypatch.setattr(api, "LIBPATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(api, "_lib", None)
    with pytest.raises(api.GTBError):
        api.load_library()


def test_pack_fields_layout():
    import numpy as np
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import pack_fields
    wl = synth.config0(seed=3, n_refs=5)
    s = synth.pack(wl.refs)
    s.mol[2] = 1
    pk = pack_fields(s)
    assert pk.n == 5 and pk.npos == s.total
    for f, a in enumerate(pk.arrays):
        assert pk.end[f] - pk.beg[f] == a.nbytes
    ins = pk.arrays[6]
    assert ins[s.offs[2]] > 0 and (ins[s.offs[[0, 1, 3, 4]]] <= 0).all()


def test_python_structs_match_the_c_header(tmp_path):
    """The ctypes mirrors of gtb_options, gtb_results, gtb_tuning,
    gtb_tuning_trial and gtb_reader_options have the C header's field offsets
    and sizes (compiled with the host C compiler)."""
    import subprocess
    from gtalign_alpha_b200.api import _COptions, _CReaderOptions, _CResults, Tuning, _CTuningTrial
    structs = (("gtb_options", _COptions), ("gtb_results", _CResults), ("gtb_tuning", Tuning),
               ("gtb_tuning_trial", _CTuningTrial), ("gtb_reader_options", _CReaderOptions))
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gtb200.h"', "int main(void) {"]
    for cname, py in structs:
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in py._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, fname))
    lines.append("return 0; }")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)])
    got = dict(l.rsplit(" ", 1) for l in subprocess.check_output([str(exe)]).decode().splitlines())
    for cname, py in structs:
        assert int(got[cname + " size"]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got["%s.%s" % (cname, fname)]) == getattr(py, fname).offset, (cname, fname)


def test_options_and_tuning_mirrors_build_on_the_host():
    """Options (keyword fields, speed presets) and Tuning convert to their C
    structs without a device."""
    from gtalign_alpha_b200.api import Options, Tuning
    o = Options(polish_steps=2, prescore=0.3)
    c = o._c()
    assert c.polish_steps == 2 and abs(c.prescore - 0.3) < 1e-7
    assert Options.speed(9)._c().nodetailedsearch == 0
    assert Options.speed(13)._c().nodetailedsearch == 1
    t = Tuning(256, 8, 0, 8192)
    assert t.as_dict() == dict(seed_chunk=256, refine_long_ctas=8, dp_cta_pairs=0, sub_pairs=8192)
    assert Tuning(**t.as_dict()).as_dict() == t.as_dict()
