"""ctypes binding of libbcc.so, the CUDA checker (C ABI in include/bcc.h).

``Checker`` mirrors the reference operator batch_cc::batch_cc<Robot>
(src/batch_cc.hh:4-6, src/batch_cc.cu:244-338): environments + edges
[E, 2, dof] + resolution in, verdicts [E, N] out (True = in collision, layout
[edge][env] as src/batch_cc.cu:131).  Errors raise ``BccError`` with the
library's message, as the reference throws std::runtime_error for bad
environments (src/batch_cc.cu:45-56).

There is no CPU fallback: if libbcc.so is missing or no CUDA device is
present, constructing a Checker raises.
"""
import ctypes
import os

import numpy as np

from .envs import BccEnvSoa

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(HERE, "libbcc.so")
ROBOTS = {"panda": 0, "fetch": 1, "baxter": 2}


def _rid(robot):
    """bcc_robot id of a robot name (an int passes through unchanged)."""
    return robot if isinstance(robot, int) else ROBOTS[robot]
ORDERS = {"plain": 0, "learned": 1}
STATUS = {0: "BCC_OK", 1: "BCC_ERR_INVALID_ARGUMENT", 2: "BCC_ERR_CUDA", 3: "BCC_ERR_NO_ENVS",
          4: "BCC_ERR_TIMEOUT", 5: "BCC_ERR_NOT_SUPPORTED", 6: "BCC_ERR_LIMIT"}


class BccError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status


class BccOpts(ctypes.Structure):
    _fields_ = [("order", ctypes.c_int32), ("use_graph", ctypes.c_int32),
                ("tile_override", ctypes.c_int32), ("learned_row_cap", ctypes.c_int32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libbcc.so not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.bcc_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int]
        L.bcc_destroy.argtypes = [vp]
        L.bcc_destroy.restype = None
        L.bcc_last_error.argtypes = [vp]
        L.bcc_last_error.restype = ctypes.c_char_p
        L.bcc_upload_envs.argtypes = [vp, ctypes.POINTER(BccEnvSoa)]
        L.bcc_check.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_int32,
                                ctypes.c_int32, ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(BccOpts)]
        L.bcc_check_device.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int32, ctypes.c_int32, vp,
                                       ctypes.POINTER(BccOpts), vp]
        L.bcc_edge_samples.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                       ctypes.c_int32, ctypes.c_int32]
        L.bcc_robot_dof.argtypes = [ctypes.c_int]
        L.bcc_measure_fp32_peak.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
        L.bcc_mlp_num_params.argtypes = []
        L.bcc_mlp_set_params.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int32]
        L.bcc_mlp_get_params.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int32]
        L.bcc_mlp_forward.argtypes = [vp, vp, ctypes.c_int32, vp, vp]
        L.bcc_mlp_gradients.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_float),
                                        ctypes.POINTER(ctypes.c_float)]
        L.bcc_mlp_train_step.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]
        L.bcc_mlp_train.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_int32, ctypes.c_int32,
                                    ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_uint64,
                                    ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        L.bcc_mlp_evaluate.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_float)]
        L.bcc_env_code.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int32]
        L.bcc_mlp_train_queued.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_int32,
                                           ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                                           ctypes.c_int32, ctypes.c_float, ctypes.c_uint64,
                                           ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                           ctypes.POINTER(ctypes.c_int64)]
        L.bcc_mlp_rank_metrics.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_int32,
                                           ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double),
                                           ctypes.c_int32]
        L.bcc_last_learned_rows.argtypes = [vp]
        L.bcc_last_learned_rows.restype = ctypes.c_int64
        L.bcc_last_learned_pairs.argtypes = [vp]
        L.bcc_last_learned_pairs.restype = ctypes.c_int64
        L.bcc_get_launch_config.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
        L.bcc_set_launch_config.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
        L.bcc_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_int32, ctypes.c_int32,
                                   ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
        L.bcc_set_profiling.argtypes = [vp, ctypes.c_int32]
        L.bcc_work_counters.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int32]
        L.bcc_stage_times.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int32]
        L.bcc_pack_envs.argtypes = [ctypes.POINTER(BccEnvSoa), ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64),
                                    ctypes.POINTER(ctypes.c_int32)]
        _lib = L
    return _lib


def exported_symbols():
    """Names declared in include/bcc.h (checked against the .so by the tests)."""
    return ["bcc_create", "bcc_destroy", "bcc_last_error", "bcc_upload_envs", "bcc_check",
            "bcc_check_device", "bcc_edge_samples", "bcc_robot_dof", "bcc_pack_envs",
            "bcc_set_profiling", "bcc_stage_times", "bcc_measure_fp32_peak", "bcc_work_counters"]


def make_opts(order="plain", use_graph=False, tile=0, row_cap=0):
    o = BccOpts()
    o.order = ORDERS[order]
    o.use_graph = int(bool(use_graph))
    o.tile_override = int(tile)
    o.learned_row_cap = int(row_cap)
    return o


class Checker:
    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        st = lib().bcc_create(ctypes.byref(self._h), device)
        if st != 0:
            raise BccError(st, "bcc_create failed (no CUDA device?)")
        self.num_envs = None

    def close(self):
        if self._h:
            lib().bcc_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _raise(self, st):
        if st != 0:
            raise BccError(st, lib().bcc_last_error(self._h).decode())

    def upload(self, envset):
        soa = envset.as_ctypes()
        self._raise(lib().bcc_upload_envs(self._h, ctypes.byref(soa)))
        self.num_envs = envset.num_envs

    def check(self, edges, resolution=32, robot="panda", order="plain", out=None, tile=0, graph=False, row_cap=0):
        """Host API: edges float32 [E, 2, dof] -> verdicts uint8 [E, num_envs].  row_cap > 0 bounds the
        learned order's MLP rows per check."""
        edges = np.ascontiguousarray(edges, np.float32)
        E = edges.shape[0]
        if out is None:
            out = np.zeros((E, self.num_envs), np.uint8)
        opts = make_opts(order, use_graph=graph, tile=tile, row_cap=row_cap)
        st = lib().bcc_check(self._h, _rid(robot), edges.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                             E, resolution, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                             ctypes.byref(opts))
        self._raise(st)
        return out

    def set_profiling(self, on=True, counters=False):
        self._raise(lib().bcc_set_profiling(self._h, (1 if on else 0) | (2 if counters else 0)))

    COUNTERS = ("pairs", "candidates", "chunks", "gate_chunks", "leaf_steps", "colliding")

    def work_counters(self):
        out = (ctypes.c_uint64 * 6)()
        if lib().bcc_work_counters(self._h, out, 6) < 0:
            raise BccError(1, "work counters are off or no check has run")
        return dict(zip(self.COUNTERS, [int(v) for v in out]))

    STAGES = ("steps", "fk", "self", "swept", "check")

    def stage_times(self):
        """Device ms of the last check's stages (stream must be synchronised)."""
        ms = (ctypes.c_float * 5)()
        n = lib().bcc_stage_times(self._h, ms, 5)
        if n < 0:
            raise BccError(1, "profiling is off or no check has run")
        return dict(zip(self.STAGES, [float(ms[i]) for i in range(n)]))

    # ---------------------------------------------------------------- MLP
    def mlp_set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        self._raise(lib().bcc_mlp_set_params(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(p)))

    def mlp_get_params(self):
        n = lib().bcc_mlp_num_params()
        p = np.zeros(n, np.float32)
        self._raise(lib().bcc_mlp_get_params(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n))
        return p

    def mlp_forward_device(self, d_x_ptr, rows, d_logits_ptr, stream=0):
        self._raise(lib().bcc_mlp_forward(self._h, ctypes.c_void_p(d_x_ptr), rows, ctypes.c_void_p(d_logits_ptr),
                                          ctypes.c_void_p(stream)))

    def mlp_gradients_device(self, d_x_ptr, d_y_ptr, rows):
        n = lib().bcc_mlp_num_params()
        g = np.zeros(n, np.float32)
        loss = ctypes.c_float(0)
        self._raise(lib().bcc_mlp_gradients(self._h, ctypes.c_void_p(d_x_ptr), ctypes.c_void_p(d_y_ptr), rows,
                                            g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(loss)))
        return g, float(loss.value)

    def mlp_train_step_device(self, d_x_ptr, d_y_ptr, rows, lr):
        loss = ctypes.c_float(0)
        self._raise(lib().bcc_mlp_train_step(self._h, ctypes.c_void_p(d_x_ptr), ctypes.c_void_p(d_y_ptr), rows,
                                             ctypes.c_float(lr), ctypes.byref(loss)))
        return float(loss.value)

    def mlp_train(self, edges, num_samples, epochs=2, batch=16384, lr=2e-3, seed=0, resolution=32, robot="panda"):
        """Train on checker-labelled samples of the uploaded envs; returns (epoch losses, positive fraction)."""
        edges = np.ascontiguousarray(edges, np.float32)
        losses = np.zeros(epochs, np.float32)
        pos = ctypes.c_float(0)
        self._raise(lib().bcc_mlp_train(self._h, _rid(robot), edges.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                        len(edges), resolution, int(num_samples), epochs, batch, ctypes.c_float(lr),
                                        ctypes.c_uint64(seed), losses.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                        ctypes.byref(pos)))
        return losses, float(pos.value)

    def mlp_train_queued(self, edges, num_samples, queue_min_items=128, epochs=2, batch=16384, lr=2e-3, seed=0,
                         resolution=32, robot="panda"):
        """Train on the segments of the pairs the learned order's probe queues (threshold queue_min_items)
        over the uploaded envs; returns (epoch losses, positive fraction, rows used)."""
        edges = np.ascontiguousarray(edges, np.float32)
        losses = np.zeros(epochs, np.float32)
        pos = ctypes.c_float(0)
        rows = ctypes.c_int64(0)
        self._raise(lib().bcc_mlp_train_queued(
            self._h, _rid(robot), edges.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(edges), resolution,
            int(queue_min_items), int(num_samples), epochs, batch, ctypes.c_float(lr), ctypes.c_uint64(seed),
            losses.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(pos), ctypes.byref(rows)))
        return losses, float(pos.value), int(rows.value)

    RANK_METRICS = ("queued_pairs", "scored_segments", "colliding_pairs", "colliding_samples", "auc",
                    "ranks_to_hit_plain", "ranks_to_hit_learned", "ranks_to_hit_perfect",
                    "ranks_walked_plain", "ranks_walked_learned", "ranks_walked_perfect", "realised_share",
                    "mispredict")

    def mlp_rank_metrics(self, edges, queue_min_items=128, resolution=32, robot="panda"):
        """Ranking quality of the current network on the learned order's population (bcc_mlp_rank_metrics)."""
        edges = np.ascontiguousarray(edges, np.float32)
        m = np.zeros(13, np.float64)
        self._raise(lib().bcc_mlp_rank_metrics(self._h, _rid(robot),
                                               edges.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(edges),
                                               resolution, int(queue_min_items),
                                               m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 13))
        return dict(zip(self.RANK_METRICS, [float(v) for v in m]))

    def mlp_evaluate(self, edges, num_samples, seed=1, resolution=32, robot="panda"):
        edges = np.ascontiguousarray(edges, np.float32)
        m = np.zeros(5, np.float32)
        self._raise(lib().bcc_mlp_evaluate(self._h, _rid(robot), edges.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                           len(edges), resolution, int(num_samples), ctypes.c_uint64(seed),
                                           m.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return dict(zip(("loss", "mispredict", "false_pos", "false_neg", "positive"), [float(v) for v in m]))

    def env_code(self):
        """The 32-value code of every uploaded environment, float32 [num_envs, 32]."""
        out = np.zeros((self.num_envs, 32), np.float32)
        self._raise(lib().bcc_env_code(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.num_envs))
        return out

    def last_learned_rows(self):
        return int(lib().bcc_last_learned_rows(self._h))

    def last_learned_pairs(self):
        return int(lib().bcc_last_learned_pairs(self._h))

    CONFIG = ("edges_per_cta", "warps", "persistent", "queue_min_items", "finish_split", "learned_mode",
              "clusters", "lanes")

    def launch_config(self):
        c = (ctypes.c_int32 * len(self.CONFIG))()
        self._raise(lib().bcc_get_launch_config(self._h, c))
        return dict(zip(self.CONFIG, list(c)))

    def set_launch_config(self, **kw):
        cfg = self.launch_config()
        cfg.update(kw)
        c = (ctypes.c_int32 * len(self.CONFIG))(*[int(cfg[k]) for k in self.CONFIG])
        self._raise(lib().bcc_set_launch_config(self._h, c))

    def autotune(self, edges, order="plain", resolution=32, robot="panda"):
        edges = np.ascontiguousarray(edges, np.float32)
        c = (ctypes.c_int32 * len(self.CONFIG))()
        self._raise(lib().bcc_autotune(self._h, _rid(robot), edges.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                       len(edges), resolution, ORDERS[order], c))
        return dict(zip(self.CONFIG, list(c)))

    def check_device(self, d_edges_ptr, num_edges, d_results_ptr, resolution=32, robot="panda",
                     order="plain", stream=0, tile=0, graph=False, row_cap=0):
        """Device API: raw device pointers (e.g. torch tensors' data_ptr()), stream-ordered."""
        opts = make_opts(order, use_graph=graph, tile=tile, row_cap=row_cap)
        st = lib().bcc_check_device(self._h, _rid(robot), ctypes.c_void_p(d_edges_ptr), num_edges,
                                    resolution, ctypes.c_void_p(d_results_ptr), ctypes.byref(opts),
                                    ctypes.c_void_p(stream))
        self._raise(st)


def edge_samples(start, end, resolution=32):
    s = np.ascontiguousarray(start, np.float32)
    e = np.ascontiguousarray(end, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    return lib().bcc_edge_samples(s.ctypes.data_as(fp), e.ctypes.data_as(fp), len(s), resolution)


def measure_fp32_peak(device=0):
    """FP32 FMA-pipe peak (TFLOP/s) of the device, from the library's probe kernel."""
    t = ctypes.c_double(0)
    st = lib().bcc_measure_fp32_peak(device, ctypes.byref(t))
    if st != 0:
        raise BccError(st, "fp32 peak probe failed")
    return t.value
