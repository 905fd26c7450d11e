"""The C-ABI library loads, exports every declared symbol, and validates on the host."""
import ctypes
import re
from pathlib import Path

import pytest

from moraine_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "moraine_b200.h"


def declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mr_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(_lib.exported_symbols()) == names


def test_version_and_sizes():
    lib = _lib.load()
    assert lib.mr_abi_version() == 4
    assert lib.mr_ks_workspace_bytes(200, 200, 17) == 200 * 200 * 20 * 4
    assert lib.mr_ks_workspace_bytes(0, 200, 17) == 0
    assert lib.mr_ds_extract_workspace_bytes(4096) == 4 * 8


@pytest.mark.parametrize("call,code", [
    (lambda L: L.mr_ks_test(None, 10, 10, 17, 1, 1, None, None, 0.05, None, None, None, 0, None), _lib.MR_ERR_INVALID),
    (lambda L: L.mr_ks_test(16, 10, 10, 600, 1, 1, None, None, 0.05, None, None, 16, 10**9, None),
     _lib.MR_ERR_UNSUPPORTED),
    (lambda L: L.mr_ks_test(16, 10, 10, 17, 1, 1, 16, None, 0.05, None, None, 16, 10, None), _lib.MR_ERR_WORKSPACE),
    (lambda L: L.mr_ks_test(16, 10, 10, 17, 1, 1, 16, None, 0.05, 16, None, 16, 10**9, None), _lib.MR_ERR_INVALID),
    (lambda L: L.mr_emi(16, 10, 17, 17, 0, 16, 16, None, 16, 10**9, None), _lib.MR_ERR_INVALID),
    (lambda L: L.mr_emi(16, 10, 1, 0, 0, 16, 16, None, 16, 10**9, None), _lib.MR_ERR_INVALID),
    (lambda L: L.mr_emi(16, 10, 17, 0, 1, 16, 16, None, 16, 10**9, None), _lib.MR_ERR_INVALID),
    (lambda L: L.mr_emperical_co_pc(16, 10, 10, 17, 16, 5, 16, 0, 4, 3, None, 0, 16, 0, None), _lib.MR_ERR_INVALID),
    (lambda L: L.mr_emperical_co_pc(16, 10, 10, 17, 16, 5, 16, 2, 3, 3, None, 0, 16, 0, None), _lib.MR_ERR_INVALID),
    (lambda L: L.mr_ds_extract(16, None, 10, 10, 9, 3, 16, 16, 100, 16, 16, 10**6, None), _lib.MR_ERR_INVALID),
])
def test_host_validation_without_gpu(call, code):
    """Bad arguments are rejected before any device work (these calls never launch)."""
    lib = _lib.load()
    assert call(lib) == code
    assert _lib.last_error()


C_HOST = r"""
#include <stdio.h>
#include <string.h>
#include "moraine_b200.h"

int main(void) {
  /* host-side paths only: no device memory, no kernel */
  if (mr_abi_version() != 4) return 1;
  if (mr_gamma_sample_bytes(MR_GAMMA_FCOMPLEX) != 8) return 2;
  if (mr_ks_workspace_bytes(100, 100, 17) == 0) return 3;
  if (mr_ds_chain_workspace_bytes(64, 64, 20, 2, 3, 1000) == 0) return 4;
  int rc = mr_ks_test(NULL, 10, 10, 17, 1, 1, NULL, NULL, 0.05, NULL, NULL, NULL, 0, NULL);
  if (rc != MR_ERR_INVALID || strlen(mr_last_error()) == 0) return 5;
  printf("ok %s\n", mr_last_error());
  return 0;
}
"""


def test_header_binds_from_plain_c(tmp_path):
    """A C99 host (no Python, no C++) compiles against the header with -pedantic -Werror,
    links the library and gets its status codes and messages."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "host.c"
    src.write_text(C_HOST)
    exe = tmp_path / "host"
    libdir = Path(_lib.load()._name).parent
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", f"-I{HEADER.parent}", str(src),
                    f"-L{libdir}", "-lmoraine_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.startswith("ok ") and "ks_test" in out.stdout


def test_kernel_timing_empty_without_launches():
    lib = _lib.load()
    lib.mr_set_kernel_timing(1)
    assert _lib.kernel_timing() == {}
    lib.mr_set_kernel_timing(0)
    assert lib.mr_kernel_timing(-1, None, None, None) == 0


def test_emi_sub_batch_cap_sizes_the_workspace():
    """A smaller EMI sub-batch lowers the workspace; a workspace sized before a larger cap
    is rejected before any device work; negative caps are invalid."""
    lib = _lib.load()
    full = lib.mr_emi_workspace_bytes(100000, 100)
    assert lib.mr_set_emi_sub_batch(4096) == 0
    try:
        small = lib.mr_emi_workspace_bytes(100000, 100)
        assert small < full / 4
        assert lib.mr_set_emi_sub_batch(0) == 0
        assert lib.mr_emi_workspace_bytes(100000, 100) == full
        assert lib.mr_emi(16, 100000, 100, 0, 0, 16, 16, None, 16, small, None) == _lib.MR_ERR_WORKSPACE
        assert lib.mr_set_emi_sub_batch(-1) == _lib.MR_ERR_INVALID
    finally:
        lib.mr_set_emi_sub_batch(0)
