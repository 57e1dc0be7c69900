"""Numpy restatement of the refinement-proposer MLP (wanniernlqg_b200/csrc/mlp.cuh) in float64.

TEST INFRASTRUCTURE ONLY: the checker for the GPU forward/backward kernels.  Weights are rounded
to BF16 (round-to-nearest-even) exactly as the device copy is; biases stay FP32.  Layout:
W1[64][8] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4.
"""
import numpy as np

F, H = 8, 64
OFF = {}
_o = 0
for name, size in (("W1", H * F), ("b1", H), ("W2", H * H), ("b2", H), ("W3", H * H), ("b3", H), ("w4", H), ("b4", 1)):
    OFF[name] = (_o, size)
    _o += size
COUNT = _o


def bf16_round(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.float32)
    bits = x.view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray):
    p = np.asarray(params, dtype=np.float32)
    out = {}
    for name, (o, size) in OFF.items():
        v = p[o:o + size]
        if name.startswith("W") or name == "w4":
            v = bf16_round(v)
        out[name] = v.astype(np.float64)
    out["W1"] = out["W1"].reshape(H, F)
    out["W2"] = out["W2"].reshape(H, H)
    out["W3"] = out["W3"].reshape(H, H)
    return out


def forward(params, x):
    q = unpack(params)
    x = np.asarray(x, dtype=np.float64).reshape(-1, F)
    h1 = np.tanh(x @ q["W1"].T + q["b1"])
    h2 = np.tanh(h1 @ q["W2"].T + q["b2"])
    h3 = np.tanh(h2 @ q["W3"].T + q["b3"])
    y = h3 @ q["w4"] + q["b4"][0]
    return y, (x, h1, h2, h3)


def loss_grad(params, x, target):
    """Mean squared error and its gradient with respect to the (BF16-rounded) weights."""
    q = unpack(params)
    y, (x, h1, h2, h3) = forward(params, x)
    t = np.asarray(target, dtype=np.float64)
    n = y.size
    loss = np.mean((y - t) ** 2)
    g = 2.0 * (y - t) / n
    grad = np.zeros(COUNT)

    def put(name, v):
        o, size = OFF[name]
        grad[o:o + size] = np.ravel(v)

    put("w4", g @ h3)
    put("b4", [g.sum()])
    dz3 = np.outer(g, q["w4"]) * (1 - h3 ** 2)
    put("W3", dz3.T @ h2)
    put("b3", dz3.sum(axis=0))
    dz2 = (dz3 @ q["W3"]) * (1 - h2 ** 2)
    put("W2", dz2.T @ h1)
    put("b2", dz2.sum(axis=0))
    dz1 = (dz2 @ q["W2"]) * (1 - h1 ** 2)
    put("W1", dz1.T @ x)
    put("b1", dz1.sum(axis=0))
    return loss, grad
