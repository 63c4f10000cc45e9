"""CPU oracle (numpy, FP64) of the gate MLP and its gradients, rounding to
BF16 at the same points as the tensor-core kernels (inputs, weights, hidden
activations and the back-propagated pre-activation gradients)."""
import numpy as np


def bf16(x):
    a = np.asarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


K = 0.7978845608028654


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(K * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(K * (x + 0.044715 * x ** 3))
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * K * (1 + 3 * 0.044715 * x * x)


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[0:256].reshape(32, 8), p[256:288], p[288:1312].reshape(32, 32), p[1312:1344], p[1344:1376], p[1376])


def forward(p, X, rounding=True):
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    W1, b1, W2, b2, w3, b3 = unpack(p)
    Xb = r(X)
    a1 = Xb @ r(W1).T + b1
    h1 = r(gelu(a1))
    a2 = h1 @ r(W2).T + b2
    h2 = r(gelu(a2))
    z = h2 @ r(w3) + b3
    return Xb, a1, h1, a2, h2, z


def loss_and_grads(p, X, Y, rounding=True, neg_weight=1.0):
    """Mean of -(Y log g + neg_weight (1-Y) log(1-g)), g = sigmoid(z), and its
    gradient in the parameter layout."""
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    W1, b1, W2, b2, w3, b3 = unpack(p)
    Xb, a1, h1, a2, h2, z = forward(p, X, rounding)
    B = len(Y)
    g = 1 / (1 + np.exp(-z))
    e = 1e-7
    loss = float(np.sum(-(Y * np.log(g + e) + neg_weight * (1 - Y) * np.log(1 - g + e)))) / B
    dz = (g * (Y + neg_weight * (1 - Y)) - Y) / B
    da2 = r(dz[:, None] * r(w3)[None, :] * gelu_grad(a2))
    dW2 = da2.T @ h1
    db2 = da2.sum(0)
    dw3 = h2.T @ dz
    db3 = dz.sum()
    dh1 = da2 @ r(W2)
    da1 = r(dh1 * gelu_grad(a1))
    dW1 = da1.T @ Xb
    db1 = da1.sum(0)
    grad = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dw3, [db3]])
    return loss, grad
