"""The drop-in boundary is a C ABI: include/cgef_b200.h compiles as strict C99 (no C++ types in any
signature), every function it declares links against libcgef_b200.so from a plain C program, and the
program runs (version and device count only; no compute call).  No GPU is needed."""
import os
import re
import shutil
import subprocess

import pytest

from cgef_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cgef_b200.h")


def declared_functions():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    return sorted(set(re.findall(r"\b(cgef_[a-z_0-9]+)\s*\(", src)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_is_c99_and_every_symbol_links(tmp_path):
    names = declared_functions()
    assert len(names) >= 40
    table = ",\n".join(f"  (void (*)(void))&{n}" for n in names)
    prog = f"""#include <stdio.h>
#include "cgef_b200.h"

typedef void (*fn)(void);
static const fn every_entry_point[] = {{
{table}
}};

int main(void) {{
  size_t n = sizeof(every_entry_point) / sizeof(every_entry_point[0]);
  for (size_t i = 0; i < n; ++i)
    if (every_entry_point[i] == NULL) return 2;
  printf("%d %d %zu\\n", (int)cgef_version(), (int)cgef_device_count(), n);
  return 0;
}}
"""
    c = tmp_path / "abi.c"
    c.write_text(prog)
    lib = _lib.library_path()
    exe = tmp_path / "abi"
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
           "-I", os.path.dirname(HEADER), str(c), "-o", str(exe), lib, f"-Wl,-rpath,{os.path.dirname(lib)}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    version, devices, n = r.stdout.split()
    assert int(version) == 1 and int(devices) >= 0 and int(n) == len(names)
