"""The MAOS-side adapter compiles against the reference's headers and links.

`maos_b200/csrc/adapter/wfs_b200.c` defines the ten functions of MAOS's GPU wavefront-sensor seam
and four of its science-evaluation seam (`cuda/sim/gpu_sim.h:35-55`) over the flat ABI of
`include/shwfs_b200.h` and `include/shwfs_evl.h`. This test compiles it with
the reference's own `maos/` and `cuda/sim/` headers (the struct layouts and field names it reads),
with warnings as errors, then links it into a shared object with no undefined symbol allowed against
`libshwfs_b200.so` and the reference's C compiled as the oracle (`oracle/_ref/libmaosref.so`: the
`error`, `dnew`, `cnew`, `lrand` and allocator routines it calls). Needs the reference tree and
no GPU.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from oracle import REF_TREE as REF
ADAPTER = os.path.join(ROOT, "maos_b200", "csrc", "adapter", "wfs_b200.c")
SEAM = ["gpu_wfsgrad_init", "gpu_wfs_init_sim", "gpu_wfsgrad_update_etf", "gpu_wfsgrad_update_ref",
        "gpu_wfsgrad_seeding", "gpu_wfsgrad_queue", "gpu_wfsgrad_sync", "gpu_save_pistat",
        "gpu_wfssurf2gpu", "gpu_atm2gpu", "gpu_perfevl_init", "gpu_perfevl_init_sim",
        "gpu_perfevl_queue", "gpu_perfevl_sync", "gpu_dmreal2gpu", "gpu_dmproj2gpu"]


@pytest.fixture(scope="module")
def adapter_so(tmp_path_factory, ref_lib):
    if not os.path.isdir(os.path.join(REF, "maos")):
        pytest.skip("reference tree absent")
    lib = os.path.join(ROOT, "maos_b200", "libshwfs_b200.so")
    if not os.path.exists(lib):
        pytest.skip("libshwfs_b200.so not built")
    d = tmp_path_factory.mktemp("adapter")
    obj, so = str(d / "wfs_b200.o"), str(d / "libadapter.so")
    cc = ["gcc", "-std=gnu11", "-fPIC", "-c", "-DHAVE_CONFIG_H", "-Wall", "-Wextra", "-Werror",
          "-Wno-unused-parameter", "-I" + os.path.join(ROOT, "oracle", "refbuild"),
          "-I" + os.path.join(REF, "maos"), "-I" + os.path.join(REF, "cuda", "sim"),
          "-I" + os.path.join(ROOT, "include"), ADAPTER, "-o", obj]
    r = subprocess.run(cc, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    ld = ["gcc", "-shared", "-o", so, obj, "-L" + os.path.join(ROOT, "oracle", "_ref"),
          "-l:libmaosref.so", "-L" + os.path.dirname(lib), "-l:libshwfs_b200.so",
          "-Wl,--no-undefined", "-lpthread", "-lm"]
    r = subprocess.run(ld, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return so


def test_adapter_defines_the_seam(adapter_so):
    out = subprocess.run(["nm", "-D", "--defined-only", adapter_so], capture_output=True,
                         text=True, check=True).stdout
    defined = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [s for s in SEAM if s not in defined]
    assert not missing, missing


def test_adapter_calls_only_declared_abi(adapter_so):
    """Every shwfs_* symbol the adapter needs is one that a header under include/ declares."""
    out = subprocess.run(["nm", "-u", adapter_so], capture_output=True, text=True, check=True).stdout
    used = {ln.split()[-1] for ln in out.splitlines() if ln.split()[-1].startswith("shwfs_")}
    inc = os.path.join(ROOT, "include")
    header = "".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    assert used, "the adapter calls no library entry point"
    for s in used:
        assert s + "(" in header, s
