"""The C ABI is plain C: include/mm_match.h compiles as strict C99 and a C
program links against libmmatch.so with it alone.

The program calls only entry points that answer without a device (round caps,
the version string, argument errors), so this runs on the CPU.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "mm_match.h"

int main(void)
{
    mm_graph *g = NULL;
    int rounds = 0;
    if (mm_max_rounds(MM_TYPE_RANDOM) != 20 || mm_max_rounds(MM_TYPE_WEIGHTED_MAXIMAL) != 255) return 1;
    if (mm_max_rounds(3) != -1) return 2;
    if (mm_graph_create(-1, NULL, 0, NULL, NULL, -1, &g) != MM_ERR_ARG || g != NULL) return 3;
    if (mm_match(NULL, MM_TYPE_RANDOM_MAXIMAL, 0u, NULL, 0, NULL, &rounds, NULL) != MM_ERR_ARG) return 4;
    if (strlen(mm_last_error()) == 0) return 5;
    if (strncmp(mm_version(), "mmatch", 6) != 0) return 6;
    printf("ok\n");
    return 0;
}
"""


def test_header_is_plain_c_and_links(mm, tmp_path):
    lib = mm.PKG / "libmmatch.so"
    if not lib.exists():
        pytest.fail("libmmatch.so is not built")
    src = tmp_path / "abi.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
                    str(src), f"-L{mm.PKG}", "-lmmatch", f"-Wl,-rpath,{mm.PKG}", "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == "ok", (p.returncode, p.stdout, p.stderr)
