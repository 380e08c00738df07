"""Oracle: the expansion-order network in NumPy float64 (test infrastructure only).

The reference has no network (it takes p from the caller, HFMM.py:55-80), so
this is not a restatement of reference code: it is the CPU statement of the
3 x 64 MLP the library trains on the GPU, against which the CUDA forward,
gradient and Adam kernels are checked.

Layout of the flat parameter vector (row-major, input index first):
W1 [in][64], b1 [64], W2 [64][64], b2 [64], W3 [64][64], b3 [64], W4 [64][out], b4 [out].
Hidden activations tanh, linear output, loss = mean over samples and outputs of
the squared error. Adam follows Kingma & Ba (2015), Algorithm 1.
"""
import numpy as np

H = 64


def shapes(n_in, n_out):
    return [("W1", (n_in, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
            ("b3", (H,)), ("W4", (H, n_out)), ("b4", (n_out,))]


def param_count(n_in, n_out):
    return sum(int(np.prod(s)) for _, s in shapes(n_in, n_out))


def unpack(P, n_in, n_out):
    out, o = {}, 0
    for name, s in shapes(n_in, n_out):
        n = int(np.prod(s))
        out[name] = P[o:o + n].reshape(s)
        o += n
    return out


def forward(P, X, n_out):
    X = np.asarray(X, np.float64)
    w = unpack(np.asarray(P, np.float64), X.shape[1], n_out)
    a1 = np.tanh(X @ w["W1"] + w["b1"])
    a2 = np.tanh(a1 @ w["W2"] + w["b2"])
    a3 = np.tanh(a2 @ w["W3"] + w["b3"])
    return a3 @ w["W4"] + w["b4"], (a1, a2, a3)


def loss_grad(P, X, T, n_out):
    """(loss, dloss/dP) of the mean squared error."""
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64).reshape(len(X), n_out)
    w = unpack(np.asarray(P, np.float64), X.shape[1], n_out)
    Y, (a1, a2, a3) = forward(P, X, n_out)
    E = Y - T
    loss = float(np.mean(E * E))
    g = 2.0 * E / E.size
    d3 = (g @ w["W4"].T) * (1 - a3 * a3)
    d2 = (d3 @ w["W3"].T) * (1 - a2 * a2)
    d1 = (d2 @ w["W2"].T) * (1 - a1 * a1)
    grads = dict(W1=X.T @ d1, b1=d1.sum(0), W2=a1.T @ d2, b2=d2.sum(0), W3=a2.T @ d3,
                 b3=d3.sum(0), W4=a3.T @ g, b4=g.sum(0))
    G = np.concatenate([grads[name].reshape(-1) for name, _ in shapes(X.shape[1], n_out)])
    return loss, G


def adam(P, X, T, n_out, steps, lr, m=None, v=None, t0=0, b1=0.9, b2=0.999, eps=1e-8):
    """`steps` full-batch Adam steps; returns (P, m, v, final loss)."""
    P = np.array(P, np.float64)
    m = np.zeros_like(P) if m is None else np.array(m, np.float64)
    v = np.zeros_like(P) if v is None else np.array(v, np.float64)
    for t in range(t0 + 1, t0 + steps + 1):
        _, g = loss_grad(P, X, T, n_out)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        P -= lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return P, m, v, loss_grad(P, X, T, n_out)[0]
