"""The MAOS-side adapter, run as the simulator runs it, against the reference's CPU frame.

`oracle/_ref/libmaosadapter.so` holds the adapter (`maos_b200/csrc/adapter/wfs_b200.c`, the ten
`gpu_*` functions of `cuda/sim/gpu_sim.h` over `libshwfs_b200.so`) and a driver that calls
`gpu_wfsgrad_init`, `gpu_atm2gpu`, `gpu_wfsgrad_queue` and `gpu_wfsgrad_sync` on the `parms_t`,
`powfs_t` and screens that the reference's own setup built. Every static array the library gets
(subaperture origins, amplitude, pixel map from `dtf.si`, nominal DTF, ETF, LLT amplitude,
matched filter, i0 sums) is the one the adapter reads from the reference's structures. The
gradients that come back in `simu->gradcl` must match the reference's own CPU frame on the same
screens within 1e-4 relative (max |dg| / max |g|), as the library's direct frames do.
"""
import ctypes as C
import os

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER_LIB = os.path.join(ROOT, "oracle", "_ref", "libmaosadapter.so")


def _adapter(ref_lib):
    if not os.path.exists(ADAPTER_LIB):
        pytest.skip("oracle/_ref/libmaosadapter.so is not built (make -C oracle adapter)")
    ref_lib.lib()  # the reference's C, which the adapter library links to, loads first
    L = C.CDLL(ADAPTER_LIB)
    L.oadp_init.restype = C.c_int
    L.oadp_init.argtypes = [C.c_int, C.c_double]
    L.oadp_frame.restype = C.c_int
    L.oadp_frame.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    return L


def _screens(cfg):
    from maos_b200.workload import build
    wl = build(cfg, device=0, seed=3, noisy=False, nx=512)
    screens, layers = wl.screens, wl.layers
    wl.close()
    return screens, layers


# the two-wavelength cases: one band per powfs.wvl, from powfs.dtf[iwvl] and etfsim[iwvl]
@pytest.mark.parametrize("cfg_name,isims,wfs", [("NGS8", (5, 6), (0,)), ("LGS30", (0, 37), (0, 3)),
                                                 ("NGS8_2WVL", (4,), (0,)), ("LGS8_N32_2WVL", (3,), (0, 1))])
def test_adapter_frames_match_reference(ref_lib, cfg_name, isims, wfs):
    from maos_b200 import configs
    from tests.helpers import grad_rel_err
    cfg = getattr(configs, cfg_name)
    screens, layers = _screens(cfg)
    r = ref_lib.RefPowfs(cfg)
    ref_lib.atm_set(screens, layers)
    A = _adapter(ref_lib)
    nwfs = A.oadp_init(0, cfg["dt"])
    assert nwfs == len(cfg["thetax"])
    g = np.zeros(nwfs * 2 * r.nsa)
    for isim in isims:
        assert A.oadp_frame(isim, 0, nwfs, g.ctypes.data_as(C.POINTER(C.c_double))) == 0
        for k in wfs:
            _, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, cfg["dt"], noisy=False)
            gk = g[k * 2 * r.nsa:(k + 1) * 2 * r.nsa]
            assert np.isfinite(gk).all()
            err = grad_rel_err(gk, g_ref)
            assert err <= 1e-4, (cfg_name, isim, k, err)


@pytest.mark.parametrize("isim", [5, 6])
def test_adapter_etf_update_matches_reference(ref_lib, isim):
    """gpu_wfsgrad_update_etf with the reference's second ETF (sodium layer 1.5 km higher) and
    coldtrat 4: frame isim blends the pair with weight (isim mod 4)/4, on both sides."""
    from maos_b200.configs import LGS30
    from tests.helpers import grad_rel_err
    screens, layers = _screens(LGS30)
    r = ref_lib.RefPowfs(LGS30)
    r.setup_etf2(1500.0, 4)
    ref_lib.atm_set(screens, layers)
    A = _adapter(ref_lib)
    nwfs = A.oadp_init(0, LGS30["dt"])
    A.oadp_update_etf()
    g = np.zeros(nwfs * 2 * r.nsa)
    assert A.oadp_frame(isim, 0, nwfs, g.ctypes.data_as(C.POINTER(C.c_double))) == 0
    for k in (0, 4):
        _, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, LGS30["dt"], noisy=False)
        err = grad_rel_err(g[k * 2 * r.nsa:(k + 1) * 2 * r.nsa], g_ref)
        assert err <= 1e-4, (isim, k, err)


def test_adapter_seeding_keys_the_noise(ref_lib):
    """gpu_wfsgrad_seeding gives each WFS one lrand() of the simulator's stream: the same stream
    seed gives the same noisy frame bit for bit, another seed another frame, and the noisy
    gradients are finite and differ from the noise-free ones."""
    from maos_b200.configs import NGS8
    from tests.helpers import grad_rel_err
    screens, layers = _screens(NGS8)
    r = ref_lib.RefPowfs(NGS8)
    ref_lib.atm_set(screens, layers)
    A = _adapter(ref_lib)
    A.oadp_seed.argtypes = [C.c_uint]
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    n = 2 * r.nsa
    g0, g1, g2, g3 = (np.zeros(n) for _ in range(4))
    A.oadp_init(0, NGS8["dt"])
    A.oadp_frame(5, 0, 1, ptr(g0))
    A.oadp_init(1, NGS8["dt"])
    A.oadp_seed(1)
    A.oadp_frame(5, 0, 1, ptr(g1))
    A.oadp_seed(1)
    A.oadp_frame(5, 0, 1, ptr(g2))
    A.oadp_seed(2)
    A.oadp_frame(5, 0, 1, ptr(g3))
    assert np.array_equal(g1, g2)
    assert not np.array_equal(g1, g3)
    assert np.isfinite(g1).all()
    assert grad_rel_err(g1, g0) > 1e-3


@pytest.mark.parametrize("pttr", [0, 1])
def test_adapter_science_matches_reference(ref_lib, pttr):
    """gpu_perfevl_init / init_sim / queue / sync on the reference's 8 m science aperture and its
    PSF grid (locfft), three directions split over two threads: simu->olep (PR, TT, PTTR) and
    simu->olmp (piston, tip, tilt) of each frame against the reference's loc_calc_ptt on its own
    ray trace, within 1e-4 relative. The PSF sums run in the same frames."""
    import math
    from maos_b200.configs import LGS30
    from maos_b200.setup import screens
    from maos_b200.workload import wind
    as2rad = math.pi / 180 / 3600
    nx, seed, dt = 1024, 7, 1 / 800
    cfg = dict(LGS30, atm=dict(LGS30["atm"], nx=nx, dx=1 / 32))
    at = cfg["atm"]
    scr = screens(nx, nx, at["dx"], at["r0"], at["L0"], at["wt"], seed)
    vx, vy = wind(cfg, seed)
    o = -nx / 2 * at["dx"]
    layers = [dict(nx=nx, ny=nx, dx=at["dx"], ox=o, oy=o, ht=float(h), vx=float(vx[i]), vy=float(vy[i]),
                   alpha=1.0) for i, h in enumerate(at["ht"])]
    ref_lib.atm_set(scr, layers)
    wvl, nembed, psfsize = [1.25e-6], [512], [128]
    e = ref_lib.RefEvl(8.0, 1.2, 1 / 32, wvl=wvl, nembed=nembed)
    dirs = [(0.0, 0.0, math.inf), (20 * as2rad, -10 * as2rad, math.inf), (5 * as2rad, 5 * as2rad, 90e3)]
    A = _adapter(ref_lib)
    dp = C.POINTER(C.c_double)
    A.oadp_evl_init.argtypes = [C.c_int, dp, dp, dp, C.c_int, dp, C.POINTER(C.c_long), C.c_int, C.c_double,
                                C.c_int]
    A.oadp_evl_frame.argtypes = [C.c_int, dp, dp]
    arr = lambda v: np.ascontiguousarray(v, dtype=np.float64)
    tx, ty, hs = (arr([d[i] for d in dirs]) for i in range(3))
    w, ps = arr(wvl), np.ascontiguousarray(psfsize, dtype=np.int64)
    ptr = lambda a: a.ctypes.data_as(dp)
    assert A.oadp_evl_init(len(dirs), ptr(tx), ptr(ty), ptr(hs), 1, ptr(w), ps.ctypes.data_as(C.POINTER(C.c_long)),
                           pttr, dt, 16) == len(dirs)
    wfe, coeff = np.zeros(3 * len(dirs)), np.zeros(3 * len(dirs))
    for isim in (3, 11):
        assert A.oadp_evl_frame(isim, ptr(wfe), ptr(coeff)) == 0
        for k, d in enumerate(dirs):
            _, wfe_r, coeff_r, _ = e.frame(*d, isim, dt, pttr=pttr, psfsize=psfsize)
            assert np.all(np.abs(wfe[3 * k:3 * k + 3] - wfe_r) <= 1e-4 * np.abs(wfe_r)), (isim, k)
            assert np.abs(coeff[3 * k:3 * k + 3] - coeff_r).max() <= 1e-4 * np.abs(coeff_r).max(), (isim, k)


def _adapter_full(ref_lib):
    A = _adapter(ref_lib)
    dp, lp = C.POINTER(C.c_double), C.POINTER(C.c_long)
    A.oadp_set_cl.argtypes = [C.c_int, C.c_int, C.POINTER(dp), lp, lp, dp, dp, dp, dp, dp, dp, C.c_double, dp]
    A.oadp_set_opdadd.argtypes = [dp]
    A.oadp_poke.argtypes = [C.c_int, C.c_double]
    return A


@pytest.mark.parametrize("cfg_name,isim", [("LGS8_N32", 9), ("NGS8", 4)])
def test_adapter_closed_loop_matches_reference(ref_lib, cfg_name, isim):
    """sim.closeloop with DM surfaces (simu->dmrealsq through gpu_dmreal2gpu), the tip/tilt mirror,
    the FSM (downlink for NGS, uplink for LGS), the telescope focus, the LGS trombone and an NCPA
    surface (powfs.opdadd through gpu_wfssurf2gpu): the adapter's gradients against the reference's
    CPU frame with the same terms (maos/wfsgrad.c:200-262, 373-377), within 1e-4 relative."""
    from maos_b200 import configs
    from tests.helpers import grad_rel_err
    from tests.test_gpu_closedloop import _mirrors
    cfg = getattr(configs, cfg_name)
    llt = bool(cfg.get("has_llt"))
    screens, layers = _screens(cfg)
    r = ref_lib.RefPowfs(cfg)
    ref_lib.atm_set(screens, layers)
    A = _adapter_full(ref_lib)
    nwfs = A.oadp_init(0, cfg["dt"])
    mir, surf = _mirrors(cfg["D"], seed=21)
    keep = [np.ascontiguousarray(x, dtype=np.float64) for x in surf]
    dp = C.POINTER(C.c_double)
    sp = (dp * len(keep))(*[k.ctypes.data_as(dp) for k in keep])
    col = lambda key, t=np.float64: np.ascontiguousarray([m[key] for m in mir], dtype=t)
    nx, ny = col("nx", np.int64), col("ny", np.int64)
    dxs, ox, oy, ht = col("dx"), col("ox"), col("oy"), col("ht")
    ttm = np.array([2.5e-7, -1.5e-7])
    fsm = np.array([[1.0e-7 * (k + 1), -6e-8 * (k + 1)] for k in range(nwfs)]).ravel()
    telfocus = 3e-9
    zoomint = np.array([1.5e-9 * (k + 1) for k in range(nwfs)])
    ptr = lambda a: a.ctypes.data_as(dp)
    lptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_long))
    assert A.oadp_set_cl(1, len(mir), sp, lptr(nx), lptr(ny), ptr(dxs), ptr(ox), ptr(oy), ptr(ht), ptr(ttm),
                         ptr(fsm), telfocus, ptr(zoomint) if llt else None) == 0
    opdadd = np.random.default_rng(22).normal(0, 2e-8, r.nsa * r.nopd ** 2)
    assert A.oadp_set_opdadd(ptr(opdadd)) == 0
    g = np.zeros(nwfs * 2 * r.nsa)
    assert A.oadp_frame(isim, 0, nwfs, ptr(g)) == 0
    for k in range(nwfs):
        f = fsm[2 * k:2 * k + 2]
        ptt = (0.0, -ttm[0] - (0 if llt else f[0]), -ttm[1] - (0 if llt else f[1]))
        ref_lib.cl_set(mir, surf, use_dm=True, ptt=ptt, focus_tel=-telfocus,
                       focus_llt=-zoomint[k] if llt else 0.0, lltptt=tuple(f) if llt else (0.0, 0.0), opdadd=opdadd)
        _, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, cfg["dt"], noisy=False)
        err = grad_rel_err(g[k * 2 * r.nsa:(k + 1) * 2 * r.nsa], g_ref)
        assert err <= 1e-4, (cfg_name, k, err)
    ref_lib.cl_set()
    A.oadp_set_opdadd(None)


def test_adapter_geometric_sensor_and_phystep(ref_lib):
    """A geometric powfs (usephy 0, gtype_sim z-tilt) returns the z-tilt of the frame's OPD
    (pts_ztilt); a physical-optics powfs with phystep 3 returns z-tilt gradients (without noise,
    cuda/sim/wfsgrad.cu:709-712) before frame 3 and physical-optics ones from it; a powfs with
    step 2 leaves simu->gradcl unset before frame 2."""
    from maos_b200.configs import NGS8
    from tests.helpers import grad_rel_err
    screens, layers = _screens(NGS8)
    r = ref_lib.RefPowfs(NGS8)
    ref_lib.atm_set(screens, layers)
    A = _adapter_full(ref_lib)
    dp = C.POINTER(C.c_double)
    n = 2 * r.nsa
    g = np.zeros(n)
    # geometric sensor (noisy, but without neasim no noise is drawn)
    assert A.oadp_poke(13, 0) == 0 and A.oadp_poke(14, 1) == 0
    A.oadp_init(1, NGS8["dt"])
    A.oadp_frame(6, 0, 1, g.ctypes.data_as(dp))
    opd, _ = ref_lib.frame_opd(r, 0, 6, NGS8["dt"])
    assert grad_rel_err(g, r.ztilt(opd)) <= 1e-4
    # physical optics from frame 3 on
    assert A.oadp_poke(13, 1) == 0 and A.oadp_poke(15, 3) == 0
    A.oadp_init(1, NGS8["dt"])
    A.oadp_frame(1, 0, 1, g.ctypes.data_as(dp))
    opd, _ = ref_lib.frame_opd(r, 0, 1, NGS8["dt"])
    assert grad_rel_err(g, r.ztilt(opd)) <= 1e-4
    A.oadp_init(0, NGS8["dt"])
    A.oadp_frame(4, 0, 1, g.ctypes.data_as(dp))
    _, g_ref, _ = ref_lib.frame_full_mt(r, 0, 4, NGS8["dt"], noisy=False)
    assert grad_rel_err(g, g_ref) <= 1e-4
    # the WFS starts at frame 2
    assert A.oadp_poke(15, 0) == 0 and A.oadp_poke(16, 2) == 0
    A.oadp_init(0, NGS8["dt"])
    g[:] = 1.0
    A.oadp_frame(1, 0, 1, g.ctypes.data_as(dp))
    assert not g.any()
    A.oadp_frame(2, 0, 1, g.ctypes.data_as(dp))
    _, g_ref, _ = ref_lib.frame_full_mt(r, 0, 2, NGS8["dt"], noisy=False)
    assert grad_rel_err(g, g_ref) <= 1e-4
    A.oadp_poke(16, 0)

