"""Many independent transforms in one CUDA-graph launch (library extension; the reference
transforms one problem per call).

    tb = TransformBatch([(plan_0, c_0), (plan_1, c_1), ...])   # plans: DevicePlan
    tb.launch()              # one graph launch on the current torch stream
    tb.outputs[i]            # (B_i, n_i) float64 tensor, written by every launch

c_i are CUDA float64 tensors (B_i, m_i) (column t = row t), read by every launch: update
them in place between launches.  branches = 0 tunes the number of concurrent graph branches
when the batch is created.
"""
import ctypes

from . import _lib as L


class TransformBatch:
    def __init__(self, items, branches=0):
        import torch
        lib = L.lib()
        self.plans = [p for p, _ in items]
        self.inputs = []
        self.outputs = []
        arr = (L.NufhtB200BatchItem * len(items))()
        for q, (plan, c) in enumerate(items):
            assert c.is_cuda and c.dtype == torch.float64 and c.is_contiguous() and c.shape[1] == plan.m
            out = torch.empty((c.shape[0], plan.n), dtype=torch.float64, device=c.device)
            self.inputs.append(c)
            self.outputs.append(out)
            arr[q] = L.NufhtB200BatchItem(plan._h.value, c.data_ptr(), plan.m, out.data_ptr(), plan.n,
                                          c.shape[0])
        h = ctypes.c_void_p()
        rc = lib.nufht_b200_batch_create(ctypes.byref(h), arr, len(items), int(branches))
        if rc != 0:
            raise RuntimeError("nufht_b200_batch_create failed (%d): %s" % (rc, L.strerror(rc)))
        self._h = h

    def launch(self, stream=None):
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.inputs[0].device)
        rc = L.lib().nufht_b200_batch_launch(self._h, ctypes.c_void_p(st.cuda_stream))
        if rc != 0:
            raise RuntimeError("nufht_b200_batch_launch failed (%d): %s" % (rc, L.strerror(rc)))
        return self.outputs

    def info(self):
        br = ctypes.c_int()
        ms = ctypes.c_float()
        nodes = ctypes.c_long()
        L.lib().nufht_b200_batch_info(self._h, ctypes.byref(br), ctypes.byref(ms), ctypes.byref(nodes))
        return {"branches": br.value, "tuned_ms": ms.value, "kernel_nodes": nodes.value}

    def close(self):
        if getattr(self, "_h", None):
            L.lib().nufht_b200_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
