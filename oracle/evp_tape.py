"""Taped FP64 reference gradient of the EVP-1D subcycle loop -- TEST
INFRASTRUCTURE ONLY.

A vectorised float64 torch (CPU) restatement of the reference's 1D kernels,
differentiated by torch autograd.  It is the checker of the hand-written
adjoint of the CUDA library, alongside central finite differences of the
C oracle.  It follows:

- stress: src/bench_v2b.F90:62-312 (strain rates :363-397, Delta, capping
  :415-437, the 12 corner relaxations :186-212, str1..8 :217-310);
- stepu: src/bench_v2b.F90:444-549;
- the loop ndte x {stress; stepu}: integration/ice_dyn_evp1d.F90:188-207,
  with str1..str8 zero at the start of the call (src/bench_v0.F90:132) and
  halo velocities held fixed.

Branches follow the forward: max(Delta, DminArea) picks one side
(torch.where); a square root of 0 gets derivative 0 (as the library's
adjoint defines it).  The forward agrees with the C oracle to rounding, not
bit for bit (torch may order sums differently).  Only tests/ use this module.
"""
from __future__ import annotations

import numpy as np
import torch

P111 = 1.0 / 9.0
P055 = P111 * 0.5
P027 = P055 * 0.5
P166 = 1.0 / 6.0
P333 = 1.0 / 3.0
P222 = 2.0 / 9.0


class _SafeSqrt(torch.autograd.Function):
    """sqrt with derivative 0 at 0."""

    @staticmethod
    def forward(ctx, x):
        y = torch.sqrt(x)
        ctx.save_for_backward(y)
        return y

    @staticmethod
    def backward(ctx, g):
        (y,) = ctx.saved_tensors
        pos = y > 0
        return torch.where(pos, g * 0.5 / torch.where(pos, y, torch.ones_like(y)),
                           torch.zeros_like(g))


ssqrt = _SafeSqrt.apply

GRAD_FIELDS = ("strength", "Cw", "forcex", "forcey")


def _t(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64))


def geometry(dxT, dyT, hte, htn, htem1, htnm1, deltaminEVP):
    """Derived geometry of a T cell (src/bench_v2b.F90:137-147)."""
    return dict(dxT=dxT, dyT=dyT,
                cxp=1.5 * htn - 0.5 * htnm1, cyp=1.5 * hte - 0.5 * htem1,
                cxm=-(1.5 * htnm1 - 0.5 * htn), cym=-(1.5 * htem1 - 0.5 * hte),
                Dmin=deltaminEVP * (dxT * dyT),
                dxhy=0.5 * (hte - htem1), dyhx=0.5 * (htn - htnm1))


def stress_point(S, c, g, strength, p):
    """One stress pass at T points without skip masks.  S: 12 stresses,
    c: (ucc, vcc, uee, vee, une, vne, use, vse), g: geometry().  Returns the
    12 updated stresses and str1..str8."""
    ucc, vcc, uee, vee, une, vne, use, vse = c
    dxT, dyT, cxp, cyp, cxm, cym = g["dxT"], g["dyT"], g["cxp"], g["cyp"], g["cxm"], g["cym"]
    div = [cyp * ucc - dyT * uee + cxp * vcc - dxT * vse,
           cym * uee + dyT * ucc + cxp * vee - dxT * vne,
           cym * une + dyT * use + cxm * vne + dxT * vee,
           cyp * use - dyT * une + cxm * vse + dxT * vcc]
    ten = [-cym * ucc - dyT * uee + cxm * vcc + dxT * vse,
           -cyp * uee + dyT * ucc + cxm * vee + dxT * vne,
           -cyp * une + dyT * use + cxp * vne - dxT * vee,
           -cym * use - dyT * une + cxp * vse - dxT * vcc]
    shr = [-cym * vcc - dyT * vee - cxm * ucc - dxT * use,
           -cyp * vee + dyT * vcc - cxm * uee - dxT * une,
           -cyp * vne + dyT * vse - cxp * une + dxT * uee,
           -cym * vse - dyT * vne - cxp * use + dxT * ucc]
    a1, d1 = p.arlx1i, p.denom1
    keep = 1.0 - a1 * p.revp
    Dmin = g["Dmin"]
    s = list(S)
    for k in range(4):
        Delta = ssqrt(div[k] * div[k] + p.e_factor * (ten[k] * ten[k] + shr[k] * shr[k]))
        m = torch.where(Delta > Dmin, Delta, Dmin)
        tmp = p.capping * (strength / m) + (1.0 - p.capping) * (strength / (Delta + Dmin))
        z = (1.0 + p.Ktens) * tmp
        r = (1.0 - p.Ktens) * tmp * Delta
        e = p.epp2i * z
        s[k] = (S[k] * keep + a1 * (z * div[k] - r)) * d1
        s[4 + k] = (S[4 + k] * keep + a1 * e * ten[k]) * d1
        s[8 + k] = (S[8 + k] * keep + a1 * 0.5 * e * shr[k]) * d1
    dxhy, dyhx = g["dxhy"], g["dyhx"]
    pn, ps, pe, pw = s[0] + s[1], s[2] + s[3], s[0] + s[3], s[1] + s[2]
    p1, p2 = (s[0] + s[2]) * P055, (s[1] + s[3]) * P055
    mn, ms, me, mw = s[4] + s[5], s[6] + s[7], s[4] + s[7], s[5] + s[6]
    m1, m2 = (s[4] + s[6]) * P055, (s[5] + s[7]) * P055
    t12n, t12s, t12e, t12w = s[8] + s[9], s[10] + s[11], s[8] + s[11], s[9] + s[10]
    t121, t122 = (s[8] + s[10]) * P111, (s[9] + s[11]) * P111
    cpne = P111 * s[0] + p2 + P027 * s[2]
    cpnw = P111 * s[1] + p1 + P027 * s[3]
    cpsw = P111 * s[2] + p2 + P027 * s[0]
    cpse = P111 * s[3] + p1 + P027 * s[1]
    cmne = P111 * s[4] + m2 + P027 * s[6]
    cmnw = P111 * s[5] + m1 + P027 * s[7]
    cmsw = P111 * s[6] + m2 + P027 * s[4]
    cmse = P111 * s[7] + m1 + P027 * s[5]
    c12ne = P222 * s[8] + t122 + P055 * s[10]
    c12nw = P222 * s[9] + t121 + P055 * s[11]
    c12sw = P222 * s[10] + t122 + P055 * s[8]
    c12se = P222 * s[11] + t121 + P055 * s[9]
    s12ew = 0.5 * dxT * (P333 * t12e + P166 * t12w)
    s12we = 0.5 * dxT * (P333 * t12w + P166 * t12e)
    s12ns = 0.5 * dyT * (P333 * t12n + P166 * t12s)
    s12sn = 0.5 * dyT * (P333 * t12s + P166 * t12n)
    spa = 0.25 * dyT * (P333 * pn + P166 * ps)
    sma = 0.25 * dyT * (P333 * mn + P166 * ms)
    spb = 0.25 * dyT * (P333 * ps + P166 * pn)
    smb = 0.25 * dyT * (P333 * ms + P166 * mn)
    spc = 0.25 * dxT * (P333 * pe + P166 * pw)
    smc = 0.25 * dxT * (P333 * me + P166 * mw)
    spd = 0.25 * dxT * (P333 * pw + P166 * pe)
    smd = 0.25 * dxT * (P333 * mw + P166 * me)
    st = [-spa - sma - s12ew + dxhy * (-cpne + cmne) + dyhx * c12ne,
          spa + sma - s12we + dxhy * (-cpnw + cmnw) + dyhx * c12nw,
          -spb - smb + s12ew + dxhy * (-cpse + cmse) + dyhx * c12se,
          spb + smb + s12we + dxhy * (-cpsw + cmsw) + dyhx * c12sw,
          -spc + smc - s12ns - dyhx * (cpne + cmne) + dxhy * c12ne,
          spc - smc - s12sn - dyhx * (cpse + cmse) + dxhy * c12se,
          -spd + smd + s12ns - dyhx * (cpnw + cmnw) + dxhy * c12nw,
          spd - smd + s12sn - dyhx * (cpsw + cmsw) + dxhy * c12sw]
    return s, st


def stepu_point(u, v, sx, sy, f, p):
    """stepu at U points without skip masks (src/bench_v2b.F90:509-544).
    sx, sy: strintx, strinty; f: dict of kvrel, uocn, vocn, waterx, watery,
    forcex, forcey, umassdti, fm, Tbu, uinit, vinit."""
    du, dv = f["uocn"] - u, f["vocn"] - v
    vrel = f["kvrel"] * ssqrt(du * du + dv * dv)
    Cb = f["Tbu"] / (ssqrt(u * u + v * v) + p.u0)
    cca = (p.brlx + p.revp) * f["umassdti"] + vrel * p.cosw + Cb
    sg = torch.copysign(torch.ones_like(f["fm"]), f["fm"])
    ccb = f["fm"] + sg * vrel * p.sinw
    ab2 = cca * cca + ccb * ccb
    cc1 = sx + f["forcex"] + vrel * f["waterx"] + f["umassdti"] * (p.brlx * u + p.revp * f["uinit"])
    cc2 = sy + f["forcey"] + vrel * f["watery"] + f["umassdti"] * (p.brlx * v + p.revp * f["vinit"])
    return (cca * cc1 + ccb * cc2) / ab2, (cca * cc2 - ccb * cc1) / ab2


def forward(pr, ndte: int, p, leaves: dict | None = None):
    """Run ndte subcycles of problem ``pr`` (a Problem1D) with parameters ``p``
    (any object with the evp1d_params fields).  ``leaves`` may hold tensors
    that replace pr's strength, Cw, forcex, forcey, uvel0, vvel0 ([na]) and
    stress0 ([12, na]).  Returns (u[na], v[na], stress[12][na]) tensors."""
    leaves = leaves or {}
    na, navel = pr.na, pr.navel
    f = pr.f
    L = lambda k: leaves[k] if k in leaves else _t(f[k])
    strength = L("strength")
    ix = {k: torch.as_tensor(np.asarray(pr.idx[k], dtype=np.int64) - 1)
          for k in ("ee", "ne", "se", "nw", "sw", "sse")}
    skipT = torch.as_tensor(np.asarray(pr.skipT) != 0)
    skipU = torch.as_tensor(np.asarray(pr.skipU) != 0)
    g = geometry(_t(f["dxT"]), _t(f["dyT"]), _t(f["HTE"]), _t(f["HTN"]), _t(f["HTEm1"]),
                 _t(f["HTNm1"]), p.deltaminEVP)
    uarear = _t(f["uarear"])
    u_list = leaves.get("uvel0", _t(pr.uvel[:na]))
    v_list = leaves.get("vvel0", _t(pr.vvel[:na]))
    fu = {k: _t(f[k]) for k in ("uocn", "vocn", "waterx", "watery", "umassdti", "fm", "Tbu")}
    fu["kvrel"] = _t(f["aiu"]) * p.rhow * L("Cw")
    fu["forcex"], fu["forcey"] = L("forcex"), L("forcey")
    fu["uinit"] = leaves.get("uvel_init", u_list)
    fu["vinit"] = leaves.get("vvel_init", v_list)
    u_halo, v_halo = _t(pr.uvel[na:navel]), _t(pr.vvel[na:navel])
    S = leaves["stress0"] if "stress0" in leaves else _t(pr.stress)
    S = [S[k] for k in range(12)]
    zero = torch.zeros(na, dtype=torch.float64)
    zero_halo = torch.zeros(navel - na, dtype=torch.float64)
    for _ in range(ndte):
        u = torch.cat([u_list, u_halo])
        v = torch.cat([v_list, v_halo])
        c = (u_list, v_list, u[ix["ee"]], v[ix["ee"]], u[ix["ne"]], v[ix["ne"]],
             u[ix["se"]], v[ix["se"]])
        Snew, st = stress_point(S, c, g, strength, p)
        S = [torch.where(skipT, S[k], Snew[k]) for k in range(12)]
        st = [torch.cat([torch.where(skipT, zero, x), zero_halo]) for x in st]
        sx = uarear * (st[0][:na] + st[1][ix["nw"]] + st[2][ix["sse"]] + st[3][ix["sw"]])
        sy = uarear * (st[4][:na] + st[5][ix["sse"]] + st[6][ix["nw"]] + st[7][ix["sw"]])
        un, vn = stepu_point(u_list, v_list, sx, sy, fu, p)
        u_list = torch.where(skipU, u_list, un)
        v_list = torch.where(skipU, v_list, vn)
    return u_list, v_list, torch.stack(S)


def loss(u, v, uobs, vobs):
    """J = sum over list points of (u-u_obs)^2 + (v-v_obs)^2."""
    return ((u - _t(uobs)) ** 2 + (v - _t(vobs)) ** 2).sum()


def gradient(pr, ndte: int, p, uobs, vobs, wrt=GRAD_FIELDS + ("uvel0", "vvel0", "stress0")):
    """Taped gradient of J: dict of numpy arrays for the fields in ``wrt``."""
    leaves = {}
    for k in wrt:
        if k == "uvel0":
            base = pr.uvel[: pr.na]
        elif k == "vvel0":
            base = pr.vvel[: pr.na]
        elif k == "stress0":
            base = pr.stress
        else:
            base = pr.f[k]
        leaves[k] = _t(np.array(base, dtype=np.float64)).requires_grad_(True)
    u, v, _ = forward(pr, ndte, p, leaves)
    J = loss(u, v, uobs, vobs)
    J.backward()
    out = {k: t.grad.numpy().copy() for k, t in leaves.items()}
    out["J"] = float(J.detach())
    out["u"] = u.detach().numpy().copy()
    out["v"] = v.detach().numpy().copy()
    return out
