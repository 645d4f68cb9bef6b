"""include/clb.h is a plain C header: a C99 and a C++11 host compile against it (syntax only) and
link against libclb.so without unresolved symbols for every entry point they name."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = r'''
#include "clb.h"
int main(void) {
    clb_domain_desc d; clb_species_desc sp; clb_thermo_desc th; clb_stats st; clb_handle* h = 0;
    (void)d; (void)sp; (void)th; (void)st;
    if (clb_create(0, 0, &h) != CLB_INVALID_ARG) return 1;
    if (clb_checkpoint_save(h, "x", CLB_CKPT_FLOW) == CLB_OK) return 1;
    if (clb_write_vti(h, CLB_FIELD_MATERIAL, 0, "x.vti") == CLB_OK) return 1;
    if (clb_set_thermo_gate(h, 0) == CLB_OK) return 1;
    return 0;
}
'''


@pytest.mark.parametrize("compiler,std,ext", [("gcc", "-std=c99", "c"), ("g++", "-std=c++11", "cpp")])
def test_header_compiles_and_links(tmp_path, compiler, std, ext):
    if shutil.which(compiler) is None:
        pytest.skip(compiler + " not found")
    src = os.path.join(tmp_path, "host." + ext)
    with open(src, "w") as f:
        f.write(SRC)
    lib = os.path.join(ROOT, "complab3d-gems_b200")
    out = os.path.join(tmp_path, "host")
    r = subprocess.run([compiler, std, "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), src, "-o", out,
                        "-L", lib, "-lclb", "-Wl,-rpath," + lib], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
