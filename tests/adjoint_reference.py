"""Plain PyTorch float64 restatement of the taped DOP853 map, for checking the
adjoint kernel.

TEST INFRASTRUCTURE.  ``replay`` runs the DOP853 step of
src/integrators/galpy/dop853.rs:425-763 (stages, solution, FSAL, the three
dense stages, rcont1..8 and the interpolant) for a recorded step sequence
(tape rows (t_old, h, y_old[6])), vectorised over particles, with the same
force formulas as the device code.  Because the step sizes come from the
tape, the result is the same discrete map the adjoint kernel differentiates,
so torch's reverse mode (autograd) and forward mode (torch.func.jvp) of
``replay`` are independent references for the kernel's gradients, and
central finite differences of ``replay`` check the frozen-step derivative.
"""

from __future__ import annotations

import math

import torch

# DOP853 tableau in Hairer's numbering (13 = FSAL stage f(y_new)).
A = {
    2: {1: 5.26001519587677318785587544488e-2},
    3: {1: 1.97250569845378994544595329183e-2, 2: 5.91751709536136983633785987549e-2},
    4: {1: 2.95875854768068491816892993775e-2, 3: 8.87627564304205475450678981324e-2},
    5: {1: 2.41365134159266685502369798665e-1, 3: -8.84549479328286085344864962717e-1,
        4: 9.24834003261792003115737966543e-1},
    6: {1: 3.7037037037037037037037037037e-2, 4: 1.70828608729473871279604482173e-1,
        5: 1.25467687566822425016691814123e-1},
    7: {1: 3.7109375e-2, 4: 1.70252211019544039314978060272e-1, 5: 6.02165389804559606850219397283e-2,
        6: -1.7578125e-2},
    8: {1: 3.70920001185047927108779319836e-2, 4: 1.70383925712239993810214054705e-1,
        5: 1.07262030446373284651809199168e-1, 6: -1.53194377486244017527936158236e-2,
        7: 8.27378916381402288758473766002e-3},
    9: {1: 6.24110958716075717114429577812e-1, 4: -3.36089262944694129406857109825e0,
        5: -8.68219346841726006818189891453e-1, 6: 2.75920996994467083049415600797e1,
        7: 2.01540675504778934086186788979e1, 8: -4.34898841810699588477366255144e1},
    10: {1: 4.77662536438264365890433908527e-1, 4: -2.48811461997166764192642586468e0,
         5: -5.90290826836842996371446475743e-1, 6: 2.12300514481811942347288949897e1,
         7: 1.52792336328824235832596922938e1, 8: -3.32882109689848629194453265587e1,
         9: -2.03312017085086261358222928593e-2},
    11: {1: -9.3714243008598732571704021658e-1, 4: 5.18637242884406370830023853209e0,
         5: 1.09143734899672957818500254654e0, 6: -8.14978701074692612513997267357e0,
         7: -1.85200656599969598641566180701e1, 8: 2.27394870993505042818970056734e1,
         9: 2.49360555267965238987089396762e0, 10: -3.0467644718982195003823669022e0},
    12: {1: 2.27331014751653820792359768449e0, 4: -1.05344954667372501984066689879e1,
         5: -2.00087205822486249909675718444e0, 6: -1.79589318631187989172765950534e1,
         7: 2.79488845294199600508499808837e1, 8: -2.85899827713502369474065508674e0,
         9: -8.87285693353062954433549289258e0, 10: 1.23605671757943030647266201528e1,
         11: 6.43392746015763530355970484046e-1},
    14: {1: 5.61675022830479523392909219681e-2, 7: 2.53500210216624811088794765333e-1,
         8: -2.46239037470802489917441475441e-1, 9: -1.24191423263816360469010140626e-1,
         10: 1.5329179827876569731206322685e-1, 11: 8.20105229563468988491666602057e-3,
         12: 7.56789766054569976138603589584e-3, 13: -8.298e-3},
    15: {1: 3.18346481635021405060768473261e-2, 6: 2.83009096723667755288322961402e-2,
         7: 5.35419883074385676223797384372e-2, 8: -5.49237485713909884646569340306e-2,
         11: -1.08347328697249322858509316994e-4, 12: 3.82571090835658412954920192323e-4,
         13: -3.40465008687404560802977114492e-4, 14: 1.41312443674632500278074618366e-1},
    16: {1: -4.28896301583791923408573538692e-1, 6: -4.69762141536116384314449447206e0,
         7: 7.68342119606259904184240953878e0, 8: 4.06898981839711007970213554331e0,
         9: 3.56727187455281109270669543021e-1, 13: -1.39902416515901462129418009734e-3,
         14: 2.9475147891527723389556272149e0, 15: -9.15095847217987001081870187138e0},
}
B = {1: 5.42937341165687622380535766363e-2, 6: 4.45031289275240888144113950566,
     7: 1.89151789931450038304281599044, 8: -5.8012039600105847814672114227,
     9: 3.1116436695781989440891606237e-1, 10: -1.52160949662516078556178806805e-1,
     11: 2.01365400804030348374776537501e-1, 12: 4.47106157277725905176885569043e-2}
D = {
    5: {1: -0.84289382761090128651353491142e1, 6: 0.56671495351937776962531783590,
        7: -0.30689499459498916912797304727e1, 8: 0.23846676565120698287728149680e1,
        9: 0.21170345824450282767155149946e1, 10: -0.87139158377797299206789907490,
        11: 0.22404374302607882758541771650e1, 12: 0.63157877876946881815570249290,
        13: -0.88990336451333310820698117400e-1, 14: 0.18148505520854727256656404962e2,
        15: -0.91946323924783554000451984436e1, 16: -0.44360363875948939664310572000e1},
    6: {1: 0.10427508642579134603413151009e2, 6: 0.24228349177525818288430175319e3,
        7: 0.16520045171727028198505394887e3, 8: -0.37454675472269020279518312152e3,
        9: -0.22113666853125306036270938578e2, 10: 0.77334326684722638389603898808e1,
        11: -0.30674084731089398182061213626e2, 12: -0.93321305264302278729567221706e1,
        13: 0.15697238121770843886131091075e2, 14: -0.31139403219565177677282850411e2,
        15: -0.93529243588444783865713862664e1, 16: 0.35816841486394083752465898540e2},
    7: {1: 0.19985053242002433820987653617e2, 6: -0.38703730874935176555105901742e3,
        7: -0.18917813819516756882830838328e3, 8: 0.52780815920542364900561016686e3,
        9: -0.11573902539959630126141871134e2, 10: 0.68812326946963000169666922661e1,
        11: -0.10006050966910838403183860980e1, 12: 0.77771377980534432092869265740,
        13: -0.27782057523535084065932004339e1, 14: -0.60196695231264120758267380846e2,
        15: 0.84320405506677161018159903784e2, 16: 0.11992291136182789328035130030e2},
    8: {1: -0.25693933462703749003312586129e2, 6: -0.15418974869023643374053993627e3,
        7: -0.23152937917604549567536039109e3, 8: 0.35763911791061412378285349910e3,
        9: 0.93405324183624310003907691704e2, 10: -0.37458323136451633156875139351e2,
        11: 0.10409964950896230045147246184e3, 12: 0.29840293426660503123344363579e2,
        13: -0.43533456590011143754432175058e2, 14: 0.96324553959188282948394950600e2,
        15: -0.39177261675615439165231486172e2, 16: -0.14972683625798562581422125276e3},
}


class LowerGamma(torch.autograd.Function):
    """gamma(s, u) = Gamma(s) P(s, u) with d/du = u^(s-1) e^-u in both modes."""

    @staticmethod
    def forward(u, s, gamma_s):
        return gamma_s * torch.special.gammainc(torch.full_like(u, s), u)

    @staticmethod
    def setup_context(ctx, inputs, output):
        u, s, _ = inputs
        ctx.save_for_backward(u)
        ctx.save_for_forward(u)
        ctx.s = s

    @staticmethod
    def backward(ctx, g):
        (u,) = ctx.saved_tensors
        return g * torch.exp((ctx.s - 1.0) * torch.log(u) - u), None, None

    @staticmethod
    def jvp(ctx, du, _ds, _dg):
        (u,) = ctx.saved_tensors
        return du * torch.exp((ctx.s - 1.0) * torch.log(u) - u)


PARAM_NAMES = {0: ("amp",), 3: ("amp",), 1: ("amp", "b"),
               2: ("mn_amp", "mn_a", "mn_b", "nfw_amp", "nfw_a", "bulge_k")}


def force(kind: int, p, const: dict, x, y, z):
    """Acceleration of potential `kind` with differentiable parameters p."""
    if kind == 0:  # galpy cylindrical Kepler
        R = torch.sqrt(x * x + y * y)
        r2 = R * R + z * z
        pw = p[0] * r2 ** -1.5
        FR = -R * pw
        return (x / R) * FR, (y / R) * FR, -z * pw
    if kind == 3:
        r2 = x * x + y * y + z * z
        ar = -p[0] / (r2 * torch.sqrt(r2))
        return ar * x, ar * y, ar * z
    if kind == 1:
        ar = -p[0] * (x * x + y * y + z * z + p[1] * p[1]) ** -1.5
        return ar * x, ar * y, ar * z
    mn_amp, mn_a, mn_b, nfw_amp, nfw_a, bulge_k = (p[i] for i in range(6))
    r2 = x * x + y * y + z * z
    r = torch.sqrt(r2)
    g = LowerGamma.apply(r2 / const["rc2"], const["s"], const["gamma_s"])
    bo = -bulge_k * g / (r2 * r)
    zeta = torch.sqrt(z * z + mn_b * mn_b)
    Aa = mn_a + zeta
    Dd = (x * x + y * y + Aa * Aa) ** -1.5
    m = torch.log(1.0 + r / nfw_a) - r / (nfw_a + r)
    ho = -nfw_amp * m / (r2 * r)
    return (bo * x - mn_amp * x * Dd + ho * x,
            bo * y - mn_amp * y * Dd + ho * y,
            bo * z - mn_amp * z * Aa / zeta * Dd + ho * z)


def potential_constants(pot) -> dict:
    s = 1.5 - 0.5 * pot.bulge_alpha
    return {"s": s, "rc2": pot.bulge_rc * pot.bulge_rc, "gamma_s": math.gamma(s) if pot.kind == 2 else 0.0}


def params_tensor(pot, dtype=torch.float64):
    return torch.tensor([float(getattr(pot, n)) for n in PARAM_NAMES[pot.kind]], dtype=dtype)


def replay(kind: int, p, const: dict, y0, tape, nacc, tgrid):
    """Trajectory (nt, N, 6) of the recorded step sequence.

    y0 (N, 6); tape (N, S, 8) rows (t_old, h, ...) of which the first nacc[i]
    are used; tgrid (N, nt) output times.  Differentiable in y0 and p.
    """
    N, S, _ = tape.shape
    nt = tgrid.shape[1]
    pos_neg = torch.where(tgrid[:, -1] - tgrid[:, 0] > 0, 1.0, -1.0).to(tgrid.dtype)
    nacc = torch.as_tensor(nacc)

    def f(q):
        ax, ay, az = force(kind, p, const, q[:, 0], q[:, 1], q[:, 2])
        return torch.stack([q[:, 3], q[:, 4], q[:, 5], ax, ay, az], dim=1)

    kidx = torch.arange(nt)
    y = y0
    res = torch.where((kidx == 0)[None, :, None], y0[:, None, :], torch.zeros((N, nt, 6), dtype=y0.dtype))
    for s in range(S):
        active = nacc > s
        if not bool(active.any()):
            break
        t_old = tape[:, s, 0]
        h = torch.where(active, tape[:, s, 1], torch.ones_like(t_old))
        hc = h[:, None]
        K = {1: f(y)}
        for i in range(2, 13):
            K[i] = f(y + hc * sum(c * K[j] for j, c in A[i].items()))
        ynew = y + hc * sum(c * K[j] for j, c in B.items())
        K[13] = f(ynew)
        for i in (14, 15, 16):
            K[i] = f(y + hc * sum(c * K[j] for j, c in A[i].items()))
        r1 = y
        r2 = ynew - y
        r3 = hc * K[1] - r2
        r4 = r2 - hc * K[13] - r3
        rr = [hc * sum(c * K[j] for j, c in D[m].items()) for m in (5, 6, 7, 8)]
        t_new = t_old + h
        pn = pos_neg[:, None]
        emit = (active[:, None] & (kidx[None, :] >= 1) & ~(pn * tgrid < pn * t_old[:, None])
                & (pn * tgrid < pn * t_new[:, None]))
        sc = torch.where(emit, (tgrid - t_old[:, None]) / h[:, None], torch.zeros_like(tgrid))[..., None]
        s1 = 1.0 - sc
        dense = (r1[:, None] + sc * (r2[:, None] + s1 * (r3[:, None] + sc * (r4[:, None] + s1 * (
            rr[0][:, None] + sc * (rr[1][:, None] + s1 * (rr[2][:, None] + sc * rr[3][:, None])))))))
        res = torch.where(emit[..., None], dense, res)
        y = torch.where(active[:, None], ynew, y)
    return res.permute(1, 0, 2)


def pad_tapes(tapes: list):
    """Stack per-particle tapes (rows, 8) into (N, S, 8) plus counts."""
    S = max(max(len(t) for t in tapes), 1)
    out = torch.zeros((len(tapes), S, 8), dtype=torch.float64)
    for i, t in enumerate(tapes):
        out[i, : len(t)] = torch.as_tensor(t)
    return out, [len(t) for t in tapes]
