"""zk_gpu — B200 (sm_100a) BN254 MSM and Fr NTT with zk-gpu's API.

Python mirror of the reference crate's public surface (src/lib.rs:1-6: gpu, group, host,
msm, ntt), over the C ABI in include/zkg.h:

    from zk_gpu import Gpu, Group, Msm, Ntt, xyzz_to_affine, xyzz_to_affine_g2, host

    gpu = Gpu()                                     # gpu::Gpu::new()
    bases = Msm.upload_bases(gpu, plain_xy)         # Msm::upload_bases
    msm = Msm(gpu, n, Msm.default_window(n))        # Msm::new
    out = msm.run(gpu, bases, gpu.buffer(scalars))  # Msm::run -> &Buffer
    xy = xyzz_to_affine(gpu.read(out, 32))          # None = infinity
    ntt = Ntt(gpu, log_n); ntt.forward(gpu, buf)    # Ntt::new / forward / inverse

Argument errors raise ZkGpuError with the reference's panic text.
"""
from ._lib import ZkGpuError, lib
from .batch import Batch
from .gpu import Buffer, Gpu
from .group import Group
from .msm import Msm, xyzz_to_affine, xyzz_to_affine_g2
from .ntt import CosetShift, Ntt, quotient
from . import host

__all__ = ["Batch", "Buffer", "CosetShift", "Gpu", "Group", "Msm", "Ntt", "ZkGpuError", "host", "lib", "quotient", "xyzz_to_affine",
           "xyzz_to_affine_g2"]
