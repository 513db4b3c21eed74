"""The C++ interface of the reference (include/glst_force.hcu, cuda_container.hcu)
compiles against this project's headers and links libglst_b200.so (CPU:
compile and link only; tests/test_gpu_cpp_shim.py runs it)."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

CLIENT = r"""
#include <cstdio>
#include <vector>
#include "glst_force.hcu"
int main(int argc, char **argv) {
  const unsigned n = 6;
  std::vector<double> x = {1, 2, 3, 11, 12, 13}, y = {1, 2, 1, 12, 11, 12}, z = {1, 1, 2, 13, 12, 11};
  std::vector<double> q = {-0.8, 0.4, 0.4, -0.8, 0.4, 0.4};
  cuda_container<double> rx(x), ry(y), rz(z), qc(q);
  for (auto *c : {&rx, &ry, &rz, &qc}) c->transfer_to_device();
  glst_force<double> glst(n, 1e-4, 20.0, 20.0, 20.0, 10.0);
  glst.assign_atoms(rx.d_array().data(), ry.d_array().data(), rz.d_array().data(), qc.d_array().data());
  glst.calc_sf(); glst.sum_rmt_sf(); glst.calc_lr_ef(); glst.calc_sr_ef(); glst.comm_ef();
  for (size_t dev = 0; dev < glst.fx().size(); dev++) glst.fx()[dev].set(0.0);
  glst.calc_ener_force(rx.d_array().data(), ry.d_array().data(), rz.d_array().data(), qc.d_array().data());
  cuda_container<double> fx, fy, fz, en;
  glst.get_ef(fx, fy, fz, en);
  double e = 0; for (double v : en.h_array()) e += 0.5 * v;
  std::printf("%.17g %.17g %.17g\n", e, glst.energy(), fx.h_array()[0]);
  return 0;
}
"""


def build_client(out_dir):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    src = os.path.join(out_dir, "client.cu")
    exe = os.path.join(out_dir, "client")
    with open(src, "w") as f:
        f.write(CLIENT)
    pkg = os.path.join(ROOT, "gauss-legendre-spherical-t_b200")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I" + os.path.join(ROOT, "include"), "-o", exe, src, "-L" + pkg, "-lglst_b200",
                    "-Xlinker", "-rpath=" + pkg], check=True, capture_output=True)
    return exe


def test_reference_interface_compiles_and_links(tmp_path, pkg):
    if not (shutil.which("nvcc") or os.path.exists("/usr/local/cuda/bin/nvcc")):
        pytest.skip("nvcc not available")
    exe = build_client(str(tmp_path))
    assert os.path.exists(exe)
