"""The C ABI from plain C: every header of include/apocharmm_c compiles on
its own as pedantic C99, and a C program (tests/c/abi_smoke.c) links the
library and drives host-side calls of each handle type, the Langevin
piston's checks included.  No device work."""
import glob
import os
import shutil
import subprocess

import pytest

from apocharmm_b200.systems import water_box, write_charmm_files

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "apocharmm_b200")
CC = shutil.which("gcc")

pytestmark = pytest.mark.skipif(CC is None, reason="gcc not found")


def test_c_headers_compile_as_c99(tmp_path):
    for h in sorted(glob.glob(os.path.join(INC, "apocharmm_c", "*.h"))):
        src = tmp_path / "one.c"
        src.write_text(f'#include "apocharmm_c/{os.path.basename(h)}"\nint main(void) {{ return 0; }}\n')
        r = subprocess.run([CC, "-std=c99", "-pedantic", "-Wall", "-Werror", "-fsyntax-only", "-I", INC,
                            str(src)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                           timeout=60)
        assert r.returncode == 0, (h, r.stdout[-2000:])


def test_c_program_links_and_runs(tmp_path):
    exe = str(tmp_path / "abi_smoke")
    r = subprocess.run([CC, "-std=c99", "-Wall", "-Werror", "-I", INC,
                        os.path.join(ROOT, "tests", "c", "abi_smoke.c"), "-L", LIBDIR, "-lapocharmm_c",
                        "-Wl,-rpath," + LIBDIR, "-o", exe], stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True, timeout=120)
    assert r.returncode == 0, r.stdout[-3000:]
    s = water_box(27, 10.0, seed=1)
    paths = write_charmm_files(s, str(tmp_path))
    r = subprocess.run([exe, paths["psf"], paths["prm"], str(tmp_path / "t.dcd")],
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:]
