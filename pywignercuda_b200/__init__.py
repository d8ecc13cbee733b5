"""B200 (sm_100a) split-operator propagators with the instance-class API of
cabrer7/PyWignerCUDA: ``GPU_Wigner2D_FFT``, ``GPU_Wigner2D_ODM2``,
``GPU_FokkerPlank2D_FFT``, ``GPU_Wigner2D_GPitaevskii`` (+ ``_Bloch``), ``GPU_Dirac2D`` and
``GPU_Dirac3D``.  The hot path is the native library ``libwigner_b200.so``
(fused FFT + phase + damping + observable kernels, JIT-specialised per
instance by NVRTC); PyTorch provides device memory and streams."""
from ._lib import (WignerError, WignerArgumentError, WignerCompileError, WignerCudaError,  # noqa: F401
                   WignerTimeoutError, WignerNonFiniteError, WignerUnsupportedError,
                   WignerMemoryError)
from .wigner2d import (Propagator_Base, GPU_Wigner2D_FFT, GPU_Wigner2D_ODM2, GPU_FokkerPlank2D_FFT,  # noqa: F401
                       GPU_Wigner2D_GPitaevskii, GPU_Wigner2D_GPitaevskii_Bloch)
from .dirac2d import GPU_Dirac2D  # noqa: F401
from .dirac3d import GPU_Dirac3D  # noqa: F401

__all__ = ['GPU_Wigner2D_FFT', 'GPU_Wigner2D_ODM2', 'GPU_FokkerPlank2D_FFT', 'GPU_Wigner2D_GPitaevskii',
           'GPU_Wigner2D_GPitaevskii_Bloch', 'GPU_Dirac2D', 'GPU_Dirac3D',
           'Propagator_Base',
           'WignerError']
