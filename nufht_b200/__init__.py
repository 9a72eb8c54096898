"""B200-native batched nonuniform fast Hankel transform.

    g[i, t] = sum_j c[j, t] J_nu(k_i r_j)

Public surface:
  nufht_b200._pynufht      drop-in for the reference's `_pynufht` module (numpy in/out)
  nufht_b200.DevicePlan    device-resident plan on CUDA tensors / device pointers
  nufht_b200.torch_ops     torch.autograd.Function with the transform's adjoint and
                           derivatives with respect to r and k
  nufht_b200.batch         many transforms in one CUDA-graph launch
"""
from ._lib import lib, strerror  # noqa: F401
from .plan import DevicePlan  # noqa: F401
