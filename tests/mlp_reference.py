"""Float64 numpy restatement of the schedule MLP (test infrastructure only):
X -> relu(X W1 + b1) -> relu(. W2 + b2) -> . W3 + b3 (logits), with the mean
over samples of the masked binary cross-entropy of the logits, and its
analytic gradient, in the library's flat parameter layout."""
import numpy as np

F, H, O = 32, 64, 7


def unpack(w):
    w = np.asarray(w, np.float64)
    i = 0
    out = []
    for fan_in, fan_out in ((F, H), (H, H), (H, O)):
        out.append(w[i:i + fan_in * fan_out].reshape(fan_in, fan_out))
        i += fan_in * fan_out
        out.append(w[i:i + fan_out])
        i += fan_out
    assert i == w.size
    return out


def forward(w, X):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    a1 = np.maximum(X @ W1 + b1, 0.0)
    a2 = np.maximum(a1 @ W2 + b2, 0.0)
    return a1, a2, a2 @ W3 + b3


def loss(w, X, Y, M):
    z = forward(w, np.asarray(X, np.float64))[2]
    per = np.maximum(z, 0.0) - z * Y + np.log1p(np.exp(-np.abs(z)))
    return float((M * per).sum() / len(X))


def gradients(w, X, Y, M):
    X = np.asarray(X, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(w)
    a1, a2, z = forward(w, X)
    d3 = M * (1.0 / (1.0 + np.exp(-z)) - Y) / len(X)
    d2 = (d3 @ W3.T) * (a2 > 0)
    d1 = (d2 @ W2.T) * (a1 > 0)
    return np.concatenate([(X.T @ d1).ravel(), d1.sum(0), (a1.T @ d2).ravel(), d2.sum(0),
                           (a2.T @ d3).ravel(), d3.sum(0)])
