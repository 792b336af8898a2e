"""Host-side description of the collision-likelihood MLP (shapes, parameter
layout, initialisation) and an FP32 reference forward pass used by tests.

The network: x[48] -> 128 -> 128 -> 128 -> 1 with ReLU; parameters flat FP32
in the order W1[48][128], b1, W2[128][128], b2, W3[128][128], b3, w4[128], b4
(include/bcc.h).  The GPU kernels run it in BF16 on tensor cores with FP32
accumulation.
"""
import numpy as np

IN, HID = 48, 128
SHAPES = [("W1", (IN, HID)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
          ("W3", (HID, HID)), ("b3", (HID,)), ("w4", (HID,)), ("b4", (1,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unflatten(p):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


def init_params(seed=0):
    """He-style initialisation, biases zero."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SHAPES:
        if name.startswith("W") or name == "w4":
            fan_in = shape[0]
            parts.append(rng.normal(0, np.sqrt(2.0 / fan_in), shape).ravel())
        else:
            parts.append(np.zeros(int(np.prod(shape))))
    return np.concatenate(parts).astype(np.float32)


def bf16_round(a):
    """Round-to-nearest-even to BF16, returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def to_bf16_bits(a):
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def forward_reference(p, x, round_acts=True):
    """FP32 reference with the kernels' BF16 rounding of weights and activations."""
    P = unflatten(p)
    h = bf16_round(x).astype(np.float64)
    for k in (1, 2, 3):
        W = bf16_round(P["W%d" % k]).astype(np.float64)
        z = h @ W + P["b%d" % k]
        h = np.maximum(z, 0)
        if round_acts and k < 3:
            h = bf16_round(h.astype(np.float32)).astype(np.float64)
    return h @ P["w4"].astype(np.float64) + float(P["b4"][0])
