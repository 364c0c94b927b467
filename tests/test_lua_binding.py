"""The Lua C module (lua-santoku-tsetlin_b200/lua/santoku_tsetlin_capi.c),
the drop-in for the reference's `santoku.tsetlin.capi`
(lib/santoku/tsetlin/capi.c:1790-1803).  Lua and the santoku rocks are not
installed here, so the binding is compiled against declaration-only
headers (tests/lua_stub: the Lua 5.4 C API as documented, and santoku-matrix's
cvec / ivec accessors with the argument lists of the reference's call
sites) with every warning an error; its object file must define only the
module opener and call nothing but Lua, santoku-matrix, libc and entry
points that libtsetlin_b200.so exports."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "lua-santoku-tsetlin_b200", "lua", "santoku_tsetlin_capi.c")
STUB = os.path.join(ROOT, "tests", "lua_stub")
LIB = os.path.join(ROOT, "lua-santoku-tsetlin_b200", "libtsetlin_b200.so")
CSRC = os.path.join(ROOT, "lua-santoku-tsetlin_b200", "csrc")

LIBC = {"fprintf", "__fprintf_chk", "memset", "strcmp", "__stack_chk_fail", "stderr",
        "_GLOBAL_OFFSET_TABLE_"}


def _symbols(path, dynamic=False):
    out = subprocess.run(["nm"] + (["-D", "--defined-only"] if dynamic else []) + [path],
                         check=True, capture_output=True, text=True).stdout
    rows = [ln.split() for ln in out.splitlines() if ln.strip()]
    return rows


@pytest.fixture(scope="module")
def obj(tmp_path_factory):
    if not shutil.which("gcc") or not shutil.which("nm"):
        pytest.skip("gcc / nm not available")
    o = str(tmp_path_factory.mktemp("lua") / "capi.o")
    for std in ("c99", "c11"):
        subprocess.run(["gcc", "-std=" + std, "-O2", "-Wall", "-Wextra", "-Werror", "-pedantic",
                        "-fPIC", "-I", STUB, "-I", os.path.join(ROOT, "include"), "-c", SRC,
                        "-o", o], check=True)
    return o


def test_binding_compiles_warning_free(obj):
    assert os.path.getsize(obj) > 0


def test_binding_defines_only_the_module_opener(obj):
    defined = [r[-1] for r in _symbols(obj) if len(r) == 3 and r[1] in "TDB"]
    assert defined == ["luaopen_santoku_tsetlin_capi"]


def test_binding_calls_only_lua_santoku_libc_and_exported_abi(obj):
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", CSRC], check=True)
    exported = {r[-1] for r in _symbols(LIB, dynamic=True)}
    undef = sorted(r[-1] for r in _symbols(obj) if len(r) == 2 and r[0] == "U")
    tm_calls = [s for s in undef if s.startswith("tm_")]
    # every reference method has its entry point behind it
    for need in ("tm_create", "tm_load", "tm_train", "tm_predict", "tm_persist",
                 "tm_persist_buf", "tm_checkpoint", "tm_restore", "tm_reconfigure",
                 "tm_restrict", "tm_type", "tm_destroy", "tm_align", "tm_last_error"):
        assert need in tm_calls, need
    assert not [s for s in tm_calls if s not in exported]
    other = [s for s in undef if not (s.startswith("tm_") or s.startswith("lua_") or
                                      s.startswith("luaL_") or s.startswith("tk_cvec_") or
                                      s.startswith("tk_ivec_") or s in LIBC)]
    assert not other, other


def test_binding_keeps_the_reference_names():
    src = open(SRC).read()
    methods = set(re.findall(r'\{"([a-z]+)", tm_lua_[a-z]+\}', src))
    # capi.c:419-431 (methods) and 1790-1795 (module functions)
    assert {"train", "predict", "destroy", "restrict", "persist", "checkpoint", "restore",
            "reconfigure", "type", "create", "load"} <= methods
    assert '"santoku_tsetlin"' in src and '"align"' in src
    assert "int luaopen_santoku_tsetlin_capi(lua_State *L)" in src
