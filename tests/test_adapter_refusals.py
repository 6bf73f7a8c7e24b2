"""The MAOS-side adapter refuses the reference options it does not serve.

A drop-in that silently ignored an option would return gradients that differ
from MAOS's without an error.  gpu_wfsgrad_init checks the simulation's
parms_t/powfs_t before it touches the GPU and calls the reference's error() for
each option the library does not serve; error() raises SIGUSR2
(sys/common.h:96, sys/mem.c:849-903) and, as in the maos executable, ends the
process, so each case runs in a child process that must die of that signal
with the adapter's message.  No GPU is used: the
refusal comes before the library creates its context.
"""
import os
import signal
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER_LIB = os.path.join(ROOT, "oracle", "_ref", "libmaosadapter.so")

CHILD = r"""
import ctypes as C, sys
sys.path.insert(0, {root!r})
from oracle import ref
from maos_b200 import configs
cfg = getattr(configs, {cfg!r})
r = ref.RefPowfs(cfg)
# the maos executable ends the process on error() (maos/maos.c:367); the library build's
# handler (lib/aolib.c:26) returns instead, so restore the default action
ref.lib().register_signal_handler(None)
L = C.CDLL({lib!r})
L.oadp_poke.argtypes = [C.c_int, C.c_double]
L.oadp_init.argtypes = [C.c_int, C.c_double]
assert L.oadp_poke({what}, {value}) == 0
sys.stdout.flush()
L.oadp_init(0, cfg["dt"])
print("NOT REFUSED")
"""

# (poke code, value, config, expected message)
CASES = [
    (1, 10, "NGS8", "wavelengths; at most"),
    (2, 3, "LGS8_N32", "sodium sublayers"),
    (3, 0, "NGS8", "one amplitude map per WFS"),
    (4, 3, "NGS8", "matched filter or CoG only"),
    (5, 0, "NGS8", "uses MOAO"),
    (6, 2.0, "NGS8", "field stop"),
    (7, 1, "NGS8", "dithers"),
    (8, 1, "NGS8", "pistatout/psfout"),
    (9, 1, "NGS8", "DM-projected turbulence"),
    (10, 0.3, "NGS8", "cubic influence function"),
    (11, 2, "NGS8", "atm.dtrat"),
    (12, 1, "NGS8", "not a Shack-Hartmann WFS"),
]


@pytest.mark.parametrize("what,value,cfg,msg", CASES, ids=[c[3].split(";")[0] for c in CASES])
def test_adapter_refuses_unserved_option(ref_lib, what, value, cfg, msg):
    if not os.path.exists(ADAPTER_LIB):
        pytest.skip("oracle/_ref/libmaosadapter.so is not built (make -C oracle adapter)")
    code = CHILD.format(root=ROOT, cfg=cfg, lib=ADAPTER_LIB, what=what, value=value)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                       env={**os.environ, "CUDA_VISIBLE_DEVICES": ""})
    out = p.stdout + p.stderr
    assert "NOT REFUSED" not in out
    assert p.returncode == -signal.SIGUSR2, (p.returncode, out[-2000:])
    assert msg in out, out[-2000:]
