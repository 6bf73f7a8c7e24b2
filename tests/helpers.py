"""Helpers shared by the tests: feed the reference's setup into a GPU context."""
from __future__ import annotations

import numpy as np

from maos_b200 import shwfs


def powfs_desc_from_ref(ref, cfg) -> dict:
    dx = ref.ptsdx()
    llt_nx = ref.llt_nx
    lltdsa = llt_nx * dx
    return dict(
        nsa=ref.nsa, nopd=ref.nopd, embfac=cfg["embfac"], notf=ref.notf,
        pixpsax=ref.pixpsax, pixpsay=ref.pixpsay,
        pixthetax=cfg["pixtheta"], pixthetay=cfg["pixtheta"], wvl=cfg["wvl"],
        dsa=cfg["dsa"], dx=dx, areascale=ref.areascale, hs=cfg["hs"],
        has_etf=int(cfg.get("has_llt", 0)), has_llt=int(cfg.get("has_llt", 0)), llt_nx=llt_nx,
        llt_ox=cfg.get("llt_ox", 0.0), llt_oy=cfg.get("llt_oy", 0.0),
        llt_origx=(dx - lltdsa) * 0.5, llt_origy=(dx - lltdsa) * 0.5,
        gradtype=cfg["phytype"], sigmatch=cfg["sigmatch"],
        cogthres=cfg.get("cogthres", 0.0), cogoff=cfg.get("cogoff", 0.0),
        rne=cfg["rne"], bkgrnd=cfg.get("bkgrnd", 0.0), bkgrndc=cfg.get("bkgrndc", 0.0),
        saat=cfg["saat"], sigtot_cog=cfg["siglev"],
    )


def context_from_ref(ref, cfg, nwfs=1, noisy=0, device=0):
    """GPU context loaded with the static data the reference setup produced."""
    from oracle.ref import si_to_taps
    ctx = shwfs.Context(device)
    ip = ctx.powfs_add(**powfs_desc_from_ref(ref, cfg))
    ox, oy = ref.ptsorig()
    ctx.powfs_set_geom(ip, ox, oy, ref.amp(), ref.saa())
    ctx.powfs_set_saasum(ip, ref.saasum())
    idx, wt = si_to_taps(ref.si_dense(0))
    ctx.powfs_set_simap(ip, idx, wt)
    if cfg.get("has_llt"):
        ctx.powfs_set_etf(ip, ref.etf())
        ctx.powfs_set_lltamp(ip, ref.lltamp())
    else:
        ctx.powfs_set_nominal(ip, ref.nominal(0))
    iw = []
    for k in range(nwfs):
        i = ctx.wfs_add(ipowfs=ip, thetax=cfg["thetax"][k], thetay=cfg["thetay"][k], hs=cfg["hs"], hc=0.0,
                        misregx=0.0, misregy=0.0, sigsim=cfg["siglev"], wvlwt=1.0, noisy=noisy)
        if cfg["phytype"] == shwfs.SHWFS_GRAD_MF:
            ctx.wfs_set_mtche(i, ref.mtche(), ref.i0sum(), ref.i0sumsum())
        iw.append(i)
    return ctx, ip, iw


def turbulent_opd(ref, seed=1, n=1024, r0=0.186, L0=30.0):
    """OPD of the powfs pupil from one seeded von Karman screen, traced by the reference."""
    from oracle.ref import genatm_simple
    scr = genatm_simple(r0, L0, -11.0 / 3.0, 1.0 / 32, n, seed)
    ox = -n / 2 / 32.0
    opd = ref.prop_layer(scr, 1.0 / 32, ox, ox, 0.0, 0.0, 0.0, np.inf, 0.0, 0.0)
    return opd, scr


def ints_tolerance_ok(ints_gpu, ints_ref, nsa, npix, rel=1e-5):
    """Per-subaperture max |difference| <= rel * subaperture total."""
    a = ints_gpu.reshape(nsa, npix)
    b = ints_ref.reshape(nsa, npix)
    tot = np.abs(b).sum(1)
    err = np.abs(a - b).max(1)
    worst = (err / np.maximum(tot, 1e-30)).max()
    return worst <= rel, worst


def grad_rel_err(g_gpu, g_ref):
    """max |difference| / max |reference| over all gradients."""
    return np.abs(g_gpu - g_ref).max() / np.abs(g_ref).max()
