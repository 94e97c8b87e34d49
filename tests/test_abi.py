"""The C ABI as a loadable library: every function include/bismit_b200.h
declares is exported by libbismit_b200.so, host-only entry points work
without a device, and errors come back as status codes with a message."""
import ctypes as C
import os
import re

import pytest

from bismit_b200 import _ffi as F, configs, map as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bismit_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^(?:int|const char\*|int32_t)\s+(bm_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("bm_area_create", "bm_area_cycle", "bm_batch_create", "bm_batch_connect", "bm_server_tick",
              "bm_tuft_cycle_static", "bm_plan_resolve", "bm_last_error"):
        assert n in names
    assert len(names) >= 45


def test_library_exports_every_declared_function():
    lib = C.CDLL(F.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_ffi_binds_every_declared_function():
    lib = F.lib()
    for n in declared_functions():
        assert getattr(lib, n).argtypes is not None or n in ("bm_last_error", "bm_version"), n


def test_plan_resolution_needs_no_device():
    lmaps, areas, _ = configs.workload("area_256")
    d = M.area_desc("v1", lmaps, areas, configs.bench_settings())
    p = F.bm_area_plan()
    lib = F.lib()
    assert lib.bm_plan_resolve(C.byref(d), 0, C.byref(p)) == F.BM_OK
    assert p.n_syns_total == 272629760
    assert p.slab_bytes % 256 == 0


def test_errors_are_status_codes_with_messages():
    lib = F.lib()
    d = M.area_desc("v1", *configs.workload("area_64")[:2], configs.bench_settings())
    d.layers[3].tufts[0].dens_per_tft = 0   # invalid scheme
    p = F.bm_area_plan()
    rc = lib.bm_plan_resolve(C.byref(d), 0, C.byref(p))
    assert rc == F.BM_ERR_INVALID
    assert lib.bm_last_error().decode()
    assert lib.bm_area_cycle(None, 1) == F.BM_ERR_INVALID
    assert lib.bm_batch_create(None, None, 0, None) == F.BM_ERR_INVALID
    assert lib.bm_server_tick(None, None) == F.BM_ERR_INVALID


def test_regrowth_adds_the_key0_buffer():
    """With regrowth on, every data layer carries one den_src_key0 byte per
    dendrite (the key-0 membership of the dendrite's source set); with it
    off, none."""
    lib = F.lib()
    on = configs.bench_settings()
    on.bits &= ~F.BM_SET_DISABLE_REGROWTH
    for s, present in ((on, True), (configs.bench_settings(), False)):
        d = M.area_desc("v1", *configs.workload("area_64")[:2], s)
        p = F.bm_area_plan()
        assert lib.bm_plan_resolve(C.byref(d), 0, C.byref(p)) == F.BM_OK
        for l in range(p.n_layers):
            L = p.layers[l]
            k = F.BUF["den_src_key0"]
            if present:
                assert L.buf_len[k] == L.n_dens
            else:
                assert L.buf_off[k] == 2 ** 64 - 1


def test_rnd_stream_is_host_computable():
    lib = F.lib()
    a = lib.bm_rnd(7, 1, 2, F.BM_RND_DEN_CYCLE, 0, 5)
    b = lib.bm_rnd(7, 1, 2, 1, 0, 5)
    assert a == b
    assert lib.bm_rnd(7, 1, 2, 1, 0, 6) != b


STRUCTS = ["bm_src_layer_desc", "bm_tuft_desc", "bm_input_src_desc", "bm_layer_desc", "bm_area_desc",
           "bm_tuft_plan", "bm_ctrl_plan", "bm_layer_plan", "bm_io_plan", "bm_filter_chain_plan", "bm_area_plan",
           "bm_tuft_form", "bm_server_stats"]


def test_ctypes_structures_match_the_header(tmp_path):
    """Every descriptor and plan structure of the ctypes mirror has the C
    compiler's size and field offsets."""
    import subprocess
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "bismit_b200.h"', "int main(void) {"]
    for name in STRUCTS:
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (name, name))
        for f, _ in getattr(F, name)._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (name, f, name, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n") if l)
    for name in STRUCTS:
        S = getattr(F, name)
        assert int(got[name]) == C.sizeof(S), name
        for f, _ in S._fields_:
            assert int(got[name + "." + f]) == getattr(S, f).offset, name + "." + f
