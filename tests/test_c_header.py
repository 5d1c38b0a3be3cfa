"""include/gpp.h is a C header: a plain C11 program that loads a host LP with
gpp_lp_from_host, presolves it and frees the summary compiles warning-free and
links against the engine library (CPU only: the program is built, not run)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "gpu-preprocessor-ijoc_b200", "gpp_b200")

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")

PROGRAM = r"""
#include <stdio.h>
#include "gpp.h"

int main(void) {
  /* A 1 x 2 LP: x0 + x1 >= 1, 0 <= x <= 1, min x0 + x1. */
  const gpp_offset row_ptr[2] = {0, 2};
  const int32_t col_idx[2] = {0, 1};
  const double val[2] = {1.0, 1.0}, c[2] = {1.0, 1.0}, l[2] = {0.0, 0.0}, u[2] = {1.0, 1.0};
  const double AL[1] = {1.0}, AU[1] = {1e300};
  gpp_host_lp host = {1, 2, 2, row_ptr, col_idx, val, c, AL, AU, l, u, 0.0};
  gpp_lp dev = {0};
  if (gpp_lp_from_host(&host, &dev) != GPP_OK) {
    fprintf(stderr, "%s\n", gpp_last_error());
    return 1;
  }
  gpp_params params;
  gpp_default_params(&params);
  gpp_summary summary;
  if (gpp_preprocess(&dev, &params, &summary) != GPP_OK) return 1;
  gpp_free_summary(&summary);
  return 0;
}
"""


def test_gpp_h_is_c11_and_links(tmp_path):
    src = tmp_path / "host_load.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "host_load"
    cmd = ["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
           "-L", LIB_DIR, "-lgpp_b200", "-Wl,-rpath," + LIB_DIR, "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert exe.exists()
