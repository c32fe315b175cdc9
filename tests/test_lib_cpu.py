"""CPU checks of the C ABI library: it builds, loads, exports every function declared in
include/stormgpu.h, and refuses to map without a GPU (there is no CPU fallback)."""
import os
import re
import subprocess

import pytest

from storm_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def built():
    build.build()
    return api.lib()


def declared_functions():
    src = open(os.path.join(ROOT, "include", "stormgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(stormgpu_[a-z_0-9]+)\s*\(", src)))


def test_exports_every_declared_symbol(built):
    names = declared_functions()
    assert len(names) >= 12
    out = subprocess.run(["nm", "-D", "--defined-only", api.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (stormgpu_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert hasattr(built, n)


def test_cli_binaries_link_the_library(built):
    for exe in ("storm-nucleotide", "storm-color"):
        path = os.path.join(build.BIN_DIR, exe)
        assert os.access(path, os.X_OK)
        ldd = subprocess.run(["ldd", path], capture_output=True, text=True).stdout
        assert "libstormgpu.so" in ldd


@pytest.mark.skipif(api.device_available() if os.path.exists(api.LIB_PATH) else False,
                    reason="a GPU is present")
def test_no_cpu_fallback(built):
    assert not api.device_available()
    with pytest.raises(api.StormError, match="GPU"):
        api.Mapper(api.params(), "####-##")


def test_invalid_seed_rejected(built):
    with pytest.raises(api.StormError, match="seed"):
        api.Mapper(api.params(), "##x#")
