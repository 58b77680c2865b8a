"""pair_style jax/mtp argument parsing, without a GPU.

PairMTPB200::settings only parses; it calls nothing in the library.  A small
program built against the LAMMPS shim (as the mini driver is) checks the
argument forms: the reference's four to six (pair_jax_mtp.cpp:228-245), the
optional precision, the trailing `rows device|host`, and the errors.
"""

import os
import subprocess

import pytest

from conftest import REPO

PS = os.path.join(REPO, "jax-mtp_b200", "pair_style")
LIBDIR = os.path.join(REPO, "jax-mtp_b200", "mtp_b200")

PROBE = r"""
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include "pair_mtp_b200.h"
#include "lammps_shim.h"
using namespace LAMMPS_NS;

struct Probe : PairMTPB200 {
  using PairMTPB200::PairMTPB200;
  void show() {
    std::printf("ok %s %d %d %.3f %d %d %d\n", mtp_path, max_atoms, max_nbr, cutoff, debug_level, precision,
                rows_on_device);
  }
};

int main(int argc, char** argv) {
  Atom atom; Neighbor neighbor; Error error; Memory memory; Comm comm; Force force; LAMMPS lmp;
  lmp.atom = &atom; lmp.neighbor = &neighbor; lmp.error = &error; lmp.memory = &memory; lmp.comm = &comm;
  lmp.force = &force;
  std::vector<std::string> a(argv + 1, argv + argc);
  std::vector<char*> p;
  for (auto& s : a) p.push_back(&s[0]);
  try {
    Probe pair(&lmp);
    pair.settings(static_cast<int>(p.size()), p.data());
    pair.show();
  } catch (const std::exception& e) {
    std::printf("error %s\n", e.what());
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    if not os.path.exists(os.path.join(LIBDIR, "libmtp_b200.so")):
        pytest.skip("libmtp_b200.so is not built")
    d = tmp_path_factory.mktemp("probe")
    src = d / "probe.cpp"
    src.write_text(PROBE)
    exe = d / "probe"
    subprocess.run(["g++", "-O0", "-std=c++17", "-I", os.path.join(PS, "shim"), "-I", os.path.join(REPO, "include"),
                    "-I", PS, "-o", str(exe), str(src), os.path.join(PS, "pair_mtp_b200.cpp"), "-L", LIBDIR,
                    "-lmtp_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return str(exe)


def _run(exe, *args):
    out = subprocess.run([exe, *args], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    return out.stdout.split()


@pytest.mark.parametrize("args,want", [
    (("m.mtp", "2000", "60", "5.0"), ["m.mtp", "2000", "60", "5.000", "0", "0", "1"]),
    (("m.mtp", "2000", "60", "5.0", "2"), ["m.mtp", "2000", "60", "5.000", "2", "0", "1"]),
    (("m.mtp", "2000", "60", "5.0", "0", "mixed"), ["m.mtp", "2000", "60", "5.000", "0", "1", "1"]),
    (("m.mtp", "2000", "60", "5.0", "0", "fp64", "rows", "host"), ["m.mtp", "2000", "60", "5.000", "0", "0", "0"]),
    (("m.mtp", "2000", "60", "5.0", "rows", "host"), ["m.mtp", "2000", "60", "5.000", "0", "0", "0"]),
    (("m.mtp", "2000", "60", "5.0", "1", "rows", "device"), ["m.mtp", "2000", "60", "5.000", "1", "0", "1"]),
])
def test_settings_forms(probe, args, want):
    out = _run(probe, *args)
    assert out[0] == "ok", out
    assert out[1:] == want


@pytest.mark.parametrize("args", [
    ("m.mtp", "2000", "60"),                                   # too few
    ("m.mtp", "2000", "60", "5.0", "0", "fp32"),               # unknown precision
    ("m.mtp", "2000", "60", "5.0", "0", "fp64", "rows", "gpu"),  # unknown rows mode
    ("m.mtp", "0", "60", "5.0"),                               # non-positive capacity
    ("m.mtp", "2000", "60", "-1.0"),                           # non-positive cutoff
])
def test_settings_errors(probe, args):
    out = _run(probe, *args)
    assert out[0] == "error", out
