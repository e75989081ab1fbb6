"""Plain torch FP64 restatement of the learned scorer (remobench_b200/csrc/rb_mlp.cu)
for checking its forward pass and gradients -- test infrastructure only.

Same function as the CUDA kernels: inputs, weights and hidden activations
rounded to BF16 at the same points (the casts pass gradients straight
through), tanh-form GELU, loss (y0 - t0)^2 + BCE-with-logits(y1, t1) averaged
over the batch; only the accumulation is FP64 instead of FP32.
"""
import math

import torch

IN, HID, OUT = 16, 64, 2
OFF = {"W1": 0, "b1": 1024, "W2": 1088, "b2": 5184, "W3": 5248, "b3": 5376}
NUM = 5378


def unpack(p):
    p = torch.as_tensor(p, dtype=torch.float64)
    W1 = p[0:1024].reshape(HID, IN)
    b1 = p[1024:1088]
    W2 = p[1088:5184].reshape(HID, HID)
    b2 = p[5184:5248]
    W3 = p[5248:5376].reshape(OUT, HID)
    b3 = p[5376:5378]
    return W1, b1, W2, b2, W3, b3


def bf16(t):
    return t.to(torch.bfloat16).to(torch.float64)


def gelu(z):
    c = math.sqrt(2.0 / math.pi)
    return 0.5 * z * (1.0 + torch.tanh(c * (z + 0.044715 * z ** 3)))


def forward(params, x):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    x = torch.as_tensor(x, dtype=torch.float64)
    xb = bf16(x)
    a1 = bf16(gelu(xb @ bf16(W1).T + b1))
    a2 = bf16(gelu(a1 @ bf16(W2).T + b2))
    return a2 @ bf16(W3).T + b3


def loss_and_grad(params, x, t):
    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = torch.as_tensor(x, dtype=torch.float64)
    t = torch.as_tensor(t, dtype=torch.float64)
    xb = bf16(x)
    a1 = bf16(gelu(xb @ bf16(W1).T + b1))
    a2 = bf16(gelu(a1 @ bf16(W2).T + b2))
    y = a2 @ bf16(W3).T + b3
    per = (y[:, 0] - t[:, 0]) ** 2 + torch.nn.functional.binary_cross_entropy_with_logits(
        y[:, 1], t[:, 1], reduction="none")
    loss = per.mean()
    loss.backward()
    return float(loss.detach()), p.grad.numpy()
