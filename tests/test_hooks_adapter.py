"""CPU check that the Mosscap-side hook adapter (include/mosscap_b200_hooks.hpp)
compiles against the reference's own Simulation type, i.e. that it is the
binding a Mosscap maintainer can add. Needs the reference sources; no GPU."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = "/root/reference/source"


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference sources not present")
def test_adapter_compiles_against_reference_simulation():
    src = """
#include "Simulation.hpp"
#include "mosscap_b200_hooks.hpp"
void install_into(Mosscap::Simulation& sim) {
    auto ctx = mosscap_b200::install(sim);
    (void)ctx;
}
"""
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "t.cpp")
        open(f, "w").write(src)
        r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-w", f"-I{REF}",
                            "-I" + os.path.join(ROOT, "oracle", "ref_shim", "include"),
                            "-I" + os.path.join(ROOT, "include"), f], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
