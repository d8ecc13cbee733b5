"""Build drop-in propagator instances the way the reference's notebooks do
(a subclass that sets attributes and calls the constructor)."""
import numpy as np

from oracle.wigner2d import WignerParams
from oracle.dirac2d import DiracParams


def wigner_instance(prm: WignerParams, W0, time_steps, skip_frames=10 ** 9, exact=False, file_name=''):
    from pywignercuda_b200 import GPU_Wigner2D_FFT, GPU_Wigner2D_ODM2, GPU_FokkerPlank2D_FFT
    from pywignercuda_b200 import _lib
    base = GPU_Wigner2D_ODM2 if prm.odm2 else (GPU_FokkerPlank2D_FFT if prm.kvn else GPU_Wigner2D_FFT)

    class Instance(base):
        constants_mode = _lib.CONST_EXACT if exact else _lib.CONST_CUDA_F

        def __init__(self):
            self.dampingFunction = prm.damping
            self.grossPitaevskiiCoefficient = 0.0
            self.fp_Damping_String = prm.fp_damping
            self.epsilon = prm.epsilon
            self.L_material = prm.L_material
            self.SetTimeTrack(prm.dt, time_steps, skip_frames, fileName=file_name)
            if prm.kvn:
                self.kinematicString = prm.kinetic
                base.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude, prm.hbar,
                              prm.mass, prm.d_theta, prm.d_lambda, prm.gamma, prm.potential,
                              prm.dpotential, normalization=prm.normalization)
            elif prm.odm2:
                base.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude, prm.hbar,
                              prm.mass, prm.d_theta, prm.d_lambda, prm.gamma, prm.weight1,
                              prm.weight2, prm.potential, prm.dpotential, prm.kinetic)
            else:
                base.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude, prm.hbar,
                              prm.mass, prm.d_theta, prm.d_lambda, prm.gamma, prm.potential,
                              prm.dpotential, prm.kinetic)
    inst = Instance()
    inst.W_init = np.array(W0, copy=True)
    return inst


def wigner_obs(inst):
    return np.stack([inst.X_average, inst.X2_average, inst.P_average, inst.P2_average,
                     inst.XP_average, inst.dPotentialdX_average, inst.PdPotentialdX_average,
                     inst.XdPotentialdX_average, inst.Hamiltonian_average, inst.negativeArea], 1)


def dirac_instance(prm: DiracParams, psi0, time_steps, skip_frames=10 ** 9, file_name='', mode='Density'):
    from pywignercuda_b200 import GPU_Dirac2D

    class Instance(GPU_Dirac2D):
        def __init__(self):
            self.mass, self.c, self.hBar = prm.mass, prm.c, prm.hbar
            self.Potential_0_String, self.Potential_1_String = prm.A0, prm.A1
            self.Potential_2_String, self.Potential_3_String = prm.A2, prm.A3
            self.fileName = file_name
            GPU_Dirac2D.__init__(self, (prm.n_x, prm.n_y), (prm.x_amplitude, prm.y_amplitude), prm.dt,
                                 time_steps, skip_frames, frameSaveMode=mode)
    inst = Instance()
    inst.Psi_init = np.array(psi0, copy=True)
    return inst


def dirac_obs(inst):
    return np.stack([inst.X_average, inst.Y_average, inst.Alpha1_average, inst.Alpha2_average,
                     inst.Beta_average, inst.KEnergy_average, inst.Potential_0_average], 1)


def gp_instance(prm: WignerParams, a_gp, W0, time_steps, skip_frames=10 ** 9, file_name=''):
    """A GPU_Wigner2D_GPitaevskii instance the way a notebook builds one."""
    from pywignercuda_b200 import GPU_Wigner2D_GPitaevskii

    class Instance(GPU_Wigner2D_GPitaevskii):
        def __init__(self):
            self.dampingFunction = prm.damping
            self.GPitaevskiiCoeff = a_gp
            self.fp_Damping_String = prm.fp_damping
            self.epsilon = prm.epsilon
            self.L_material = prm.L_material
            self.SetTimeTrack(prm.dt, time_steps, skip_frames, fileName=file_name)
            GPU_Wigner2D_GPitaevskii.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude,
                                              prm.hbar, prm.mass, prm.d_theta, prm.d_lambda, prm.gamma,
                                              prm.potential, prm.dpotential, prm.kinetic)
    inst = Instance()
    inst.W_init = np.array(W0, copy=True)
    return inst


def bloch_instance(prm: WignerParams, a_gp, W0, time_steps, file_name=''):
    """A GPU_Wigner2D_GPitaevskii_Bloch instance the way a notebook builds one."""
    from pywignercuda_b200 import GPU_Wigner2D_GPitaevskii_Bloch

    class Instance(GPU_Wigner2D_GPitaevskii_Bloch):
        def __init__(self):
            self.GPitaevskiiCoeff = a_gp
            self.SetTimeTrack(prm.dt, time_steps, 10 ** 9, fileName=file_name)
            GPU_Wigner2D_GPitaevskii_Bloch.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude,
                                                    prm.hbar, prm.mass, prm.potential, prm.kinetic)
    inst = Instance()
    inst.W_init = np.array(W0, copy=True)
    return inst


def dirac3d_instance(prm, psi0, time_steps, skip_frames=10 ** 9, file_name='', mode='Density', constants_mode=None):
    """A GPU_Dirac3D instance the way a notebook builds one."""
    from pywignercuda_b200 import GPU_Dirac3D

    class Instance(GPU_Dirac3D):
        def __init__(self):
            self.mass, self.c, self.hBar = prm.mass, prm.c, prm.hbar
            self.Potential_0_String, self.Potential_1_String = prm.A0, prm.A1
            self.Potential_2_String, self.Potential_3_String = prm.A2, prm.A3
            self.fileName = file_name
            self.Compute_Ehrenfest_P = True
            GPU_Dirac3D.__init__(self, (prm.n_x, prm.n_y, prm.n_z), (prm.x_amplitude, prm.y_amplitude,
                                                                     prm.z_amplitude),
                                 prm.dt, time_steps, skip_frames, frameSaveMode=mode)
    if constants_mode is not None:
        Instance.constants_mode = constants_mode
    inst = Instance()
    inst.Psi_init = np.array(psi0, copy=True)
    return inst


def dirac3d_obs(inst):
    return np.stack([inst.X_average, inst.Y_average, inst.Z_average, inst.Alpha1_average, inst.Alpha2_average,
                     inst.Alpha3_average, inst.Potential_0_average, inst.Px_average, inst.Py_average,
                     inst.Pz_average, inst.K_Energy_average, inst.Norm_average], 1)
