"""PyTorch fp32 reference of the learned corrector's MLP (the parameter layout
of MPM_CORRECTOR_PARAMS in include/mpm_b200.h).  The inputs after
normalisation, the weights and the hidden activations are rounded to bf16
where the tensor-core inference rounds them; the rounding passes gradients
straight through, as the training kernel's fp32 backward pass does."""
import numpy as np
import torch

IN, HID, OUT = 16, 64, 3
OFF = {}
_o = 0
for _name, _size in (("in_mean", IN), ("in_inv_std", IN), ("out_std", OUT), ("W1", HID * IN), ("b1", HID),
                     ("W2", HID * HID), ("b2", HID), ("W3", OUT * HID), ("b3", OUT)):
    OFF[_name] = (_o, _size)
    _o += _size
NPARAMS = _o  # 5478


def split(w):
    """Named views of a flat parameter vector (numpy or torch)."""
    out = {}
    for name, (o, n) in OFF.items():
        v = w[o:o + n]
        if name == "W1":
            v = v.reshape(HID, IN)
        elif name == "W2":
            v = v.reshape(HID, HID)
        elif name == "W3":
            v = v.reshape(OUT, HID)
        out[name] = v
    return out


def _bf16(x):
    return x + (x.to(torch.bfloat16).to(torch.float32) - x).detach()


def forward(w, x):
    """w: flat fp32 torch tensor (may require grad), x: (n, 16) fp32 -> (n, 3)."""
    p = split(w)
    xn = _bf16((x - p["in_mean"]) * p["in_inv_std"])
    h1 = _bf16(torch.nn.functional.gelu(xn @ _bf16(p["W1"]).T + p["b1"], approximate="tanh"))
    h2 = _bf16(torch.nn.functional.gelu(h1 @ _bf16(p["W2"]).T + p["b2"], approximate="tanh"))
    return (h2 @ _bf16(p["W3"]).T + p["b3"]) * p["out_std"]


def loss_and_grad(w_np, feats, targs):
    """Mean squared error of the scaled targets and its gradient (fp32)."""
    w = torch.tensor(w_np, dtype=torch.float32, requires_grad=True)
    x = torch.tensor(feats, dtype=torch.float32)
    t = torch.tensor(targs, dtype=torch.float32)
    p = split(w)
    y = forward(w, x) / p["out_std"].detach()
    loss = ((y - t / p["out_std"].detach()) ** 2).mean()
    loss.backward()
    return float(loss), w.grad.numpy().copy()


def random_params(seed, feats=None, targs=None):
    """Parameters with hidden weights of unit gain and a normalisation taken
    from data (or unit)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NPARAMS, np.float32)
    p = split(w)
    p["in_mean"][:] = 0 if feats is None else feats.mean(0)
    p["in_inv_std"][:] = 1 if feats is None else 1.0 / np.maximum(feats.std(0), 1e-6)
    p["out_std"][:] = 1 if targs is None else np.sqrt((targs ** 2).mean(0))
    p["W1"][:] = rng.normal(0, 1 / np.sqrt(IN), (HID, IN))
    p["b1"][:] = rng.normal(0, 0.1, HID)
    p["W2"][:] = rng.normal(0, 1 / np.sqrt(HID), (HID, HID))
    p["b2"][:] = rng.normal(0, 0.1, HID)
    p["W3"][:] = rng.normal(0, 1 / np.sqrt(HID), (OUT, HID))
    p["b3"][:] = rng.normal(0, 0.1, OUT)
    return w
