"""CPU float64 restatement of the learned dispatcher's MLP -- TEST INFRASTRUCTURE.

Forward and backward of the 16 -> 64 -> 64 -> 3 ReLU network that
tribit_b200/csrc/model.cu runs on the GPU, written with numpy in float64 so
the GPU's FP32 gradients can be checked against it. Parameter layout follows
include/tribit.h: W1[16][64], b1[64], W2[64][64], b2[64], W3[64][3], b3[3];
norm = in_mean[16], in_std[16], out_mean[3], out_std[3]. Loss = mean over
rows and outputs of the squared error on normalised targets.
"""
import numpy as np

SIZES = [("W1", (16, 64)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)), ("W3", (64, 3)), ("b3", (3,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    out, off = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = p[off:off + k].reshape(shape)
        off += k
    return out


def forward_backward(params, norm, x, y):
    """-> (normalised predictions, loss, flat gradient) in float64."""
    P = unpack(params)
    norm = np.asarray(norm, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    xn = (x - norm[0:16]) / norm[16:32]
    z1 = xn @ P["W1"] + P["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ P["W2"] + P["b2"]
    h2 = np.maximum(z2, 0)
    out = h2 @ P["W3"] + P["b3"]
    t = (y - norm[32:35]) / norm[35:38]
    e = out - t
    n = x.shape[0]
    loss = float(np.mean(e * e))
    dy = 2.0 * e / (3 * n)
    g = {"W3": h2.T @ dy, "b3": dy.sum(0)}
    dz2 = (dy @ P["W3"].T) * (z2 > 0)
    g["W2"] = h1.T @ dz2
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ P["W2"].T) * (z1 > 0)
    g["W1"] = xn.T @ dz1
    g["b1"] = dz1.sum(0)
    flat = np.concatenate([g[name].ravel() for name, _ in SIZES])
    return out, loss, flat


def predict(params, norm, x):
    """Denormalised predictions (what tribit_model_predict returns)."""
    out, _, _ = forward_backward(params, norm, x, np.zeros((np.asarray(x).shape[0], 3)))
    norm = np.asarray(norm, dtype=np.float64)
    return out * norm[35:38] + norm[32:35]
