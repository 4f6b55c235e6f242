"""NumPy restatement of the band proposer's network and its gradient (test only).

The network of poa_b200/csrc/proposer.cu: three Conv1d(k=3, 64 channels,
zero padding, ReLU) over 32 position bins as im2col products, a mean pool
over the bins, Linear(64, 64) + ReLU, Linear(64, 4); outputs de-standardised
as o * std + mean; training loss the mean squared error of the standardised
outputs. Parameters are laid out as poa_prop_get_weights returns them:
W1[64][3*8] b1 W2[64][3*64] b2 W3[64][3*64] b3 W4[64][64] b4 W5[4][64] b5,
then 12 extras (output mean[4], output std[4], plan margins).

With ``bf16=True`` every value the kernels store as BF16 is rounded the way
they round it (round to nearest even): the inputs, the weights as GEMM
operands, the activations after bias and ReLU, the pooled vector, and on the
backward side the output-gradient and the masked activation gradients;
products accumulate in float32. With ``bf16=False`` everything is float64,
for finite-difference checks of the gradient formulas themselves.
"""
import numpy as np

T, CIN, CH, KW, OUT = 32, 8, 64, 3, 4
SHAPES = [("W1", (CH, KW * CIN)), ("b1", (CH,)), ("W2", (CH, KW * CH)), ("b2", (CH,)),
          ("W3", (CH, KW * CH)), ("b3", (CH,)), ("W4", (CH, CH)), ("b4", (CH,)), ("W5", (OUT, CH)), ("b5", (OUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)
NEXTRA = 12


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(w):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(w[o:o + n]).reshape(shape)
        o += n
    return out


def im2col(x, C):
    """x [n*T][C] -> [n*T][3*C]: row r, column k*C + c = x[r + k - 1][c] inside the read's bins."""
    R = x.shape[0]
    t = np.arange(R) % T
    out = np.zeros((R, KW * C), dtype=x.dtype)
    for k in range(KW):
        tt = t + k - 1
        ok = (tt >= 0) & (tt < T)
        src = np.clip(np.arange(R) + k - 1, 0, R - 1)
        out[:, k * C:(k + 1) * C] = np.where(ok[:, None], x[src], 0)
    return out


def col2im(dxc, C):
    """Adjoint of im2col: dy[r][c] = sum_k dxc[r - k + 1][k*C + c] inside the read's bins."""
    R = dxc.shape[0]
    t = np.arange(R) % T
    out = np.zeros((R, C), dtype=dxc.dtype)
    for k in range(KW):
        tt = t - k + 1
        ok = (tt >= 0) & (tt < T)
        src = np.clip(np.arange(R) - k + 1, 0, R - 1)
        out += np.where(ok[:, None], dxc[src, k * C:(k + 1) * C], 0)
    return out


def forward(w, X, use_bf16=True):
    """Standardised outputs [n][4] and the activations the backward pass needs."""
    ft = np.float32 if use_bf16 else np.float64
    rnd = bf16 if use_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    p = {k: np.asarray(v, dtype=ft) for k, v in unpack(w).items()}
    Wb = {k: (rnd(v) if k.startswith("W") else v) for k, v in p.items()}
    n = X.shape[0]
    x0 = rnd(np.asarray(X, dtype=ft).reshape(n * T, CIN))
    a = {"n": n}
    a["xc1"] = im2col(x0, CIN)
    a["y1"] = rnd(np.maximum(a["xc1"] @ Wb["W1"].T + p["b1"], 0))
    a["xc2"] = im2col(a["y1"], CH)
    a["y2"] = rnd(np.maximum(a["xc2"] @ Wb["W2"].T + p["b2"], 0))
    a["xc3"] = im2col(a["y2"], CH)
    a["y3"] = rnd(np.maximum(a["xc3"] @ Wb["W3"].T + p["b3"], 0))
    a["h"] = rnd(a["y3"].reshape(n, T, CH).sum(axis=1) * ft(1.0 / T))
    a["z"] = rnd(np.maximum(a["h"] @ Wb["W4"].T + p["b4"], 0))
    o = a["z"] @ Wb["W5"].T + p["b5"]
    return o, a, Wb


def predict(w, X, use_bf16=True):
    """Raw (de-standardised) outputs, as poa_prop_predict returns them."""
    o, _, _ = forward(w, X, use_bf16)
    ex = np.asarray(w[NPARAM:NPARAM + NEXTRA], dtype=o.dtype)
    return o * ex[4:8] + ex[0:4]


def loss_and_gradient(w, X, Y, use_bf16=True):
    """Mean squared error of the standardised outputs and its parameter gradient
    (NPARAM values in the parameter layout), as poa_prop_gradient computes them."""
    ft = np.float32 if use_bf16 else np.float64
    rnd = bf16 if use_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    o, a, Wb = forward(w, X, use_bf16)
    ex = np.asarray(w[NPARAM:NPARAM + NEXTRA], dtype=ft)
    yt = (np.asarray(Y, dtype=ft) - ex[0:4]) / ex[4:8]
    n = a["n"]
    d = o - yt
    scale = ft(1.0 / (n * OUT))
    loss = float((d * d * scale).sum())
    g = {}
    dob = rnd(2 * d * scale)
    g["W5"] = dob.T @ a["z"]
    g["b5"] = dob.sum(axis=0)
    dzb = rnd((dob @ Wb["W5"]) * (a["z"] > 0))
    g["W4"] = dzb.T @ a["h"]
    g["b4"] = dzb.sum(axis=0)
    dh = dzb @ Wb["W4"]
    dy3 = rnd(np.repeat(dh * ft(1.0 / T), T, axis=0) * (a["y3"] > 0))
    g["W3"] = dy3.T @ a["xc3"]
    g["b3"] = dy3.sum(axis=0)
    dy2 = rnd(col2im(dy3 @ Wb["W3"], CH) * (a["y2"] > 0))
    g["W2"] = dy2.T @ a["xc2"]
    g["b2"] = dy2.sum(axis=0)
    dy1 = rnd(col2im(dy2 @ Wb["W2"], CH) * (a["y1"] > 0))
    g["W1"] = dy1.T @ a["xc1"]
    g["b1"] = dy1.sum(axis=0)
    return loss, np.concatenate([np.asarray(g[k], dtype=np.float64).ravel() for k, _ in SHAPES])


def random_problem(seed, n):
    """Weights (He-uniform, small random biases, identity standardisation) and a batch."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NPARAM + NEXTRA)
    o = 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        if name.startswith("W"):
            lim = np.sqrt(6.0 / shape[1])
            w[o:o + k] = rng.uniform(-lim, lim, k)
        else:
            w[o:o + k] = rng.uniform(-0.1, 0.1, k)
        o += k
    w[NPARAM + 4:NPARAM + 8] = 1.0
    w[NPARAM + 8:NPARAM + 10] = 1.0
    w[NPARAM + 10] = 8.0
    w[NPARAM + 11] = 65536.0
    X = rng.uniform(0.0, 1.0, (n, T, CIN))
    Y = rng.normal(0.0, 1.0, (n, OUT))
    return w, X, Y
