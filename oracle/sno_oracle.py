"""FP64 CPU oracle of the spectral neural operator (SNO) warm start (TEST INFRASTRUCTURE ONLY).

The reference has no learned component; this is the numpy restatement of the network
the library trains and evaluates on the device (cfft_sno_*), written on the FULL grid
with plain numpy FFTs so that it shares no arithmetic with the device path, which works
on the stride-L subgrid and the spectral ASU through the library's own KRFFT.

Network (all fields real and symmetric under the group's operations):

- Input channels a(x), C_IN = 5 + 2 * len(REFLECTIONS):
  (chiN - 21) / 9, (f - 0.4) / 0.1, a one-hot of the group over GROUPS, and for each
  reflection h_j the symmetrised plane waves
  (1/|G|) sum_g cos(2 pi h_j . (R_g x_f + t_g)), the same with sin,
  at fractional physical coordinates x_f = x / N + s (s = find_optimal_shift's shift,
  (R_g, t_g) the unshifted operations), so the features are the same functions of
  position on every grid.
- Lift: v_0 = W_lift a + b_lift (WIDTH channels).
- LAYERS Fourier layers: z_l = W_l v_l + b_l + S_l(v_l), v_{l+1} = gelu(z_l) (identity for
  the last layer), with the spectral convolution
  S(v)^(h) = W_spec[class(h)] v^(h) for h inside the box |h_c,i| <= MODES - 1 (h_c the
  wrapped index of get_k_vector) and 0 outside; class(h) enumerates the sorted absolute
  components (a >= b >= c), so W_spec is one real WIDTH x WIDTH matrix per class.  Real
  matrices keep fields real (W(-h) = W(h)); the class is invariant under every cubic
  point operation, so S keeps fields symmetric.
- Projection: out = W_p2 gelu(W_p1 v_L + b_p1) + b_p2, 2 channels;
  w_A = chiN (1 - f) + chiN out_0, w_B = chiN f + chiN out_1.
- Loss: mean over samples, both channels and grid points of (out - target)^2 with
  target = ((w_A, w_B) - homogeneous) / chiN.
- gelu(x) = x Phi(x) (exact, erf form).

`bf16_mode=True` rounds, as the device does, the weights to bfloat16 and the inputs of
the tensor-core channel products (the activations entering the 1x1 layer products and
the first projection, and the gradients entering their transposes) to bfloat16; the
weight gradients take the unrounded activations, as the device's FP32 reductions do;
everything else is FP64 here.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

from . import krfft_oracle as O

GROUPS = (229, 230, 221)           # one-hot order: Im-3m, Ia-3d, Pm-3m
REFLECTIONS = ((1, 0, 0), (1, 1, 0), (1, 1, 1), (2, 0, 0), (2, 1, 0), (2, 1, 1), (2, 2, 0), (3, 1, 0))
WIDTH, MODES, LAYERS, HIDDEN = 32, 12, 4, 64
C_IN = 5 + 2 * len(REFLECTIONS)


def class_table(modes=MODES):
    """Class id of (a, b, c), a >= b >= c >= 0, a < modes: lexicographic enumeration."""
    tab = -np.ones((modes, modes, modes), dtype=np.int64)
    k = 0
    for a in range(modes):
        for b in range(a + 1):
            for c in range(b + 1):
                tab[a, b, c] = k
                k += 1
    return tab, k


CLASS_TAB, N_CLASS = class_table()


def mode_class(hc):
    """Class of wrapped indices hc (..., 3); -1 outside the retained box."""
    s = -np.sort(-np.abs(np.asarray(hc, dtype=np.int64)), axis=-1)
    inside = s[..., 0] < MODES
    cls = np.full(s.shape[:-1], -1, dtype=np.int64)
    cls[inside] = CLASS_TAB[s[inside, 0], s[inside, 1], s[inside, 2]]
    return cls


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def init_params(seed=0):
    """Seeded initial weights (FP64): uniform in +-1/sqrt(fan_in) for the channel maps,
    spectral weights uniform in +-1/(WIDTH * sqrt(N_CLASS)) scaled like the FNO default."""
    rng = np.random.default_rng(seed)

    def lin(o, i):
        b = 1.0 / np.sqrt(i)
        return rng.uniform(-b, b, (o, i)), rng.uniform(-b, b, o)

    p = {}
    p["lift_W"], p["lift_b"] = lin(WIDTH, C_IN)
    for l in range(LAYERS):
        p[f"W{l}"], p[f"b{l}"] = lin(WIDTH, WIDTH)
        p[f"S{l}"] = rng.uniform(0.0, 1.0, (N_CLASS, WIDTH, WIDTH)) / (WIDTH * WIDTH) * 4.0
    p["p1_W"], p["p1_b"] = lin(HIDDEN, WIDTH)
    p["p2_W"], p["p2_b"] = lin(2, HIDDEN)
    return p


PARAM_ORDER = (["lift_W", "lift_b"] + [k for l in range(LAYERS) for k in (f"W{l}", f"b{l}", f"S{l}")]
               + ["p1_W", "p1_b", "p2_W", "p2_b"])


def flatten(p):
    return np.concatenate([np.asarray(p[k], dtype=np.float64).ravel() for k in PARAM_ORDER])


def unflatten(v, like=None):
    like = like or init_params(0)
    out, o = {}, 0
    for k in PARAM_ORDER:
        n = like[k].size
        out[k] = np.asarray(v[o:o + n], dtype=np.float64).reshape(like[k].shape)
        o += n
    return out


def features(sg, N, chiN, f, ops_unshifted, shift):
    """Input channels (C_IN, N1, N2, N3) on the full grid, arrays indexed [x, y, z]."""
    N = tuple(N)
    X = O._all_coords(N).astype(np.float64)            # (3, Npts), column-major point order
    xf = X / np.asarray(N, dtype=np.float64)[:, None] + np.asarray(shift, dtype=np.float64)[:, None]
    ch = [np.full(X.shape[1], (chiN - 21.0) / 9.0), np.full(X.shape[1], (f - 0.4) / 0.1)]
    ch += [np.full(X.shape[1], 1.0 if sg == g else 0.0) for g in GROUPS]
    for h in REFLECTIONS:
        hv = np.asarray(h, dtype=np.float64)
        c = np.zeros(X.shape[1])
        s = np.zeros(X.shape[1])
        for op in ops_unshifted:
            ph = 2 * np.pi * (hv @ (op.Rm.astype(np.float64) @ xf + (op.tv / np.asarray(N))[:, None]))
            c += np.cos(ph)
            s += np.sin(ph)
        ch += [c / len(ops_unshifted), s / len(ops_unshifted)]
    return np.stack([v.reshape(N, order="F") for v in ch])


def _class_grid(N):
    ax = [np.arange(n) for n in N]
    hc = [np.where(a >= n - n // 2, a - n, a) for a, n in zip(ax, N)]
    H = np.stack(np.meshgrid(*hc, indexing="ij"), axis=-1)
    return mode_class(H)


def _chan(W, x):
    """Channel map: (o, i) x (S, i, ...) -> (S, o, ...)."""
    return np.einsum("oi,si...->so...", W, x)


class SNO:
    """Forward / backward of the network on full grids (S samples of one group and N)."""

    def __init__(self, params, bf16_mode=False):
        self.bf = bf16_mode
        r = bf16 if bf16_mode else (lambda x: np.asarray(x, dtype=np.float64))
        self.p = {k: (r(v) if (k.endswith("W") or k.startswith("W") or k.startswith("S")) else np.asarray(v, float))
                  for k, v in params.items()}
        self._cls = {}

    def _q(self, x):
        return bf16(x) if self.bf else x

    def _spec(self, Wc, v, N, transpose=False):
        cls = self._cls.setdefault(tuple(N), _class_grid(N))
        V = np.fft.fftn(v, axes=(-3, -2, -1))
        out = np.zeros_like(V)
        m = cls >= 0
        Wm = Wc[cls[m]]                                 # (Nm, o, i)
        if transpose:
            Wm = np.swapaxes(Wm, 1, 2)
        out[..., m] = np.einsum("moi,sim->som", Wm, V[..., m])
        return np.real(np.fft.ifftn(out, axes=(-3, -2, -1))), V

    def forward(self, a):
        """a: (S, C_IN, N1, N2, N3) -> out (S, 2, N...) and the cache for backward."""
        p, N = self.p, a.shape[2:]
        c = {"a": a}
        v = _chan(p["lift_W"], a) + p["lift_b"][None, :, None, None, None]
        for l in range(LAYERS):
            c[f"v{l}"] = v
            s, _ = self._spec(p[f"S{l}"], v, N)
            z = _chan(p[f"W{l}"], self._q(v)) + p[f"b{l}"][None, :, None, None, None] + s
            c[f"z{l}"] = z
            v = gelu(z) if l < LAYERS - 1 else z
        c["vL"] = v
        hp = _chan(p["p1_W"], self._q(v)) + p["p1_b"][None, :, None, None, None]
        c["hp"] = hp
        hgel = gelu(hp)
        c["h"] = hgel
        out = _chan(p["p2_W"], hgel) + p["p2_b"][None, :, None, None, None]
        return out, c

    def loss(self, out, target):
        return float(np.mean((out - target) ** 2))

    def backward(self, out, target, c):
        """Gradients of loss(out, target) for every parameter (same keys as params)."""
        p, N = self.p, out.shape[2:]
        g = {}
        red = (0, 2, 3, 4)
        go = 2.0 * (out - target) / out.size
        g["p2_W"] = np.einsum("soxyz,shxyz->oh", go, c["h"])
        g["p2_b"] = go.sum(axis=red)
        gh = _chan(p["p2_W"].T, go) * gelu_grad(c["hp"])
        g["p1_W"] = np.einsum("soxyz,sixyz->oi", gh, c["vL"])
        g["p1_b"] = gh.sum(axis=red)
        gv = _chan(p["p1_W"].T, self._q(gh))
        for l in reversed(range(LAYERS)):
            gz = gv * gelu_grad(c[f"z{l}"]) if l < LAYERS - 1 else gv
            v = c[f"v{l}"]
            g[f"W{l}"] = np.einsum("soxyz,sixyz->oi", gz, v)
            g[f"b{l}"] = gz.sum(axis=red)
            sT, G = self._spec(p[f"S{l}"], gz, N, transpose=True)
            V = np.fft.fftn(v, axes=(-3, -2, -1))
            cls = self._cls[tuple(N)]
            m = cls >= 0
            prod = np.einsum("som,sim->moi", G[..., m], np.conj(V[..., m])).real / np.prod(N)
            gS = np.zeros_like(p[f"S{l}"])
            np.add.at(gS, cls[m], prod)
            g[f"S{l}"] = gS
            gv = _chan(p[f"W{l}"].T, self._q(gz)) + sT
        g["lift_W"] = np.einsum("soxyz,sixyz->oi", gv, c["a"])
        g["lift_b"] = gv.sum(axis=red)
        return g


def target_from_w(wA, wB, chiN, f):
    """Normalised network target of SCFT fields: ((w_A, w_B) - homogeneous) / chiN."""
    return np.stack([(wA - chiN * (1.0 - f)) / chiN, (wB - chiN * f) / chiN])


def w_from_output(out, chiN, f):
    return chiN * (1.0 - f) + chiN * out[0], chiN * f + chiN * out[1]
