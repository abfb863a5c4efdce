"""Build-system guards (CPU only).

The library is linked from an explicit source list, and a link in which two
objects define the same weak ``sc::`` symbol (two explicit instantiations of
one template) is refused, because the linker would keep one of them silently.
"""
import importlib.util
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "spams-devel_b200")


def _build_mod():
    spec = importlib.util.spec_from_file_location("sc_build_mod", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


SRC = """
namespace sc {
template <typename T> int launch_thing(T x) { return (int)x + %d; }
template int launch_thing<float>(float);
}
"""


def _obj(tmp_path, name, k):
    src = tmp_path / f"{name}.cpp"
    src.write_text(SRC % k)
    obj = tmp_path / f"{name}.o"
    subprocess.run(["g++", "-c", str(src), "-o", str(obj)], check=True)
    return str(obj)


def test_source_list_matches_csrc():
    b = _build_mod()
    srcs = b.sources()
    assert all(os.path.exists(s) for s in srcs)
    assert len(srcs) == len(set(srcs))


def test_duplicate_weak_instantiation_refused(tmp_path):
    b = _build_mod()
    a = _obj(tmp_path, "a", 1)
    c = _obj(tmp_path, "c", 2)
    assert any(s.startswith("_ZN2sc") for s in b._weak_host_symbols(a))
    b.check_duplicate_weak([a])
    with pytest.raises(RuntimeError, match="two objects"):
        b.check_duplicate_weak([a, c])
