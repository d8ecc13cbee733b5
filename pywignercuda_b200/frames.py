"""Frame and observable files in the reference's layout, written off the compute stream.

The reference writes every ``skipFrames``-th state with a blocking ``gpuarray.get()`` into an h5py file
(``save_Frame`` GPU_Wigner2D_FFT.py:660-663; ``save_Spinor`` / ``save_Density`` GPU_Dirac2D.py:703-737),
opens the file with the grid description (``WriteHDF5_variables`` GPU_Wigner2D_FFT.py:844-857;
GPU_Dirac2D.py:981-1009) and closes it with the Ehrenfest arrays (GPU_Wigner2D_FFT.py:1936-1959).
Notebooks read it back with ``WignerFunctionFromFile`` / ``LoadEhrenfestFromFile`` (:908-940) and
``load_Density`` / ``load_Spinor`` (GPU_Dirac2D.py:739-769).

Here a frame costs the compute stream one device-to-device copy into a snapshot buffer.  A copy
stream waits for that copy and moves the snapshot into pinned host memory; a writer thread waits for
the host copy, forms the frame (the density for Dirac ``'Density'`` mode) and writes it.  ``depth``
snapshot / pinned pairs are cycled; the host thread that captures waits only when all of them are
still being written.

The file is HDF5 through h5py when h5py is importable.  Without it the same keys go into
``fileName + '.npz'`` (one array per key; group paths kept as ``'Ehrenfest/X_Ehrenfest'``), and the
loaders read either.
"""
import os
import queue
import threading

import numpy as np

try:                                   # HDF5 output is optional (h5py may be absent)
    import h5py as _h5py
except ImportError:                    # pragma: no cover - depends on the image
    _h5py = None


def _key(k):
    return str(k).lstrip('/')


class NpzFile:
    """Write-once key store with the subset of the h5py ``File`` interface the
    propagators use (``f[key] = value``, ``create_dataset``, ``close``)."""

    def __init__(self, path):
        self.path = path
        self._data = {}

    def __setitem__(self, key, value):
        k = _key(key)
        if k in self._data:
            raise ValueError('dataset %r already exists' % k)
        self._data[k] = np.array(value, copy=True)

    def create_dataset(self, key, data):
        self[key] = data

    def __contains__(self, key):
        return _key(key) in self._data

    def __getitem__(self, key):
        return self._data[_key(key)]

    def close(self):
        with open(self.path, 'wb') as fh:
            np.savez(fh, **self._data)


class _NpzReader:
    def __init__(self, path):
        self._z = np.load(path, allow_pickle=False)

    def __getitem__(self, key):
        return self._z[_key(key)]

    def __contains__(self, key):
        return _key(key) in self._z.files

    def keys(self):
        return list(self._z.files)

    def close(self):
        self._z.close()


def open_write(fileName):
    """A fresh output file (an existing one is removed first, as ``Run`` does)."""
    path = fileName if _h5py is not None else fileName + '.npz'
    try:
        os.remove(path)
    except OSError:
        pass
    if _h5py is not None:
        return _h5py.File(path, 'w')
    return NpzFile(path)


def open_read(fileName):
    """The file ``open_write(fileName)`` made: HDF5 if h5py can read it, else the ``.npz`` twin."""
    if _h5py is not None and os.path.exists(fileName):
        return _h5py.File(fileName, 'r')
    if os.path.exists(fileName + '.npz'):
        return _NpzReader(fileName + '.npz')
    raise FileNotFoundError(fileName if _h5py is not None else fileName + '.npz')


def append(fileName, key, value):
    """Add (or replace) one dataset in a closed file, as ``Run_ExitedState1`` adds ``W_1``."""
    if _h5py is not None:
        with _h5py.File(fileName, 'a') as f:
            if _key(key) in f:
                del f[_key(key)]
            f[_key(key)] = value
        return
    path = fileName + '.npz'
    with np.load(path, allow_pickle=False) as z:
        data = {k: z[k] for k in z.files}
    data[_key(key)] = np.array(value, copy=True)
    with open(path, 'wb') as fh:
        np.savez(fh, **data)


def read(fileName, key):
    f = open_read(fileName)
    try:
        return np.array(f[key][...])
    finally:
        f.close()


def copy_frame(frame):
    """A private copy of a frame (an array, or a tuple of arrays)."""
    if isinstance(frame, tuple):
        return tuple(np.array(a, copy=True) for a in frame)
    return np.array(frame, copy=True)


class FrameWriter:
    """Asynchronous frame capture for one state shape.

    ``capture(key, state, stream)`` snapshots ``state`` (a contiguous CUDA tensor) on ``stream`` and
    returns; the write happens later on the writer thread as ``sink[...]`` assignments made by
    ``emit(sink, key, host_array)``.  ``keep`` (a dict, may be None) receives a private copy of each
    host frame as ``emit`` formed it.  ``close()`` waits for every pending frame and re-raises the
    first error of the writer thread."""

    def __init__(self, like, sink, emit, keep=None, depth=3):
        import torch
        self._torch = torch
        self.sink, self.emit, self.keep = sink, emit, keep
        self.device = like.device
        self.copy_stream = torch.cuda.Stream(device=self.device)
        self.snap = [torch.empty_like(like) for _ in range(depth)]
        self.host = [torch.empty(like.shape, dtype=like.dtype, pin_memory=True) for _ in range(depth)]
        self.free = queue.Queue()
        for s in range(depth):
            self.free.put(s)
        self.todo = queue.Queue()
        self.error = None
        self.thread = threading.Thread(target=self._loop, name='frame-writer', daemon=True)
        self.thread.start()
        self.n_frames = 0

    def capture(self, key, state, stream=None):
        torch = self._torch
        if self.error is not None:
            raise self.error
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        slot = self.free.get()
        with torch.cuda.stream(st):
            self.snap[slot].copy_(state)                  # device to device on the compute stream
            snapped = torch.cuda.Event()
            snapped.record(st)
        self.copy_stream.wait_event(snapped)
        with torch.cuda.stream(self.copy_stream):
            self.host[slot].copy_(self.snap[slot], non_blocking=True)
            done = torch.cuda.Event()
            done.record(self.copy_stream)
        self.todo.put((key, slot, done))
        self.n_frames += 1

    def _loop(self):
        while True:
            item = self.todo.get()
            if item is None:
                self.todo.task_done()
                return
            key, slot, done = item
            try:
                if self.error is None:
                    done.synchronize()
                    frame = self.emit(self.sink, key, self.host[slot].numpy())
                    if self.keep is not None:
                        self.keep[key] = copy_frame(frame)
            except Exception as exc:                       # surfaced by capture() / close()
                self.error = exc
            finally:
                self.free.put(slot)
                self.todo.task_done()

    def close(self):
        if self.thread.is_alive():
            self.todo.put(None)
            self.thread.join()
        if self.error is not None:
            raise self.error


# ---------------------------------------------------------------- Wigner layout
def wigner_header(f, inst):
    """``WriteHDF5_variables`` (GPU_Wigner2D_FFT.py:844-857) and the ``Hamiltonian``
    dataset ``Run`` adds (:1766)."""
    f['dx'], f['dtheta'], f['dp'], f['dlambda'] = inst.dX, inst.dTheta, inst.dP, inst.dLambda
    f['x_gridDIM'], f['p_gridDIM'] = inst.X_gridDIM, inst.P_gridDIM
    f['x_min'], f['x_max'] = -inst.X_amplitude, inst.X_amplitude - inst.dX
    f['p_min'], f['p_max'] = -inst.P_amplitude, inst.P_amplitude - inst.dP
    f['lambda_min'], f['lambda_max'] = inst.Lambda_range.min(), inst.Lambda_range.max()
    f['dt'], f['timeSteps'], f['skipFrames'] = inst.dt, inst.timeSteps, inst.skipFrames
    f.create_dataset('Hamiltonian', data=np.real(inst.Hamiltonian))


def wigner_frame(f, key, W):
    """``save_Frame``: the complex state under its step index."""
    f.create_dataset(str(key), data=W)
    return W


EHRENFEST_KEYS = (('X_Ehrenfest', 'X_average'), ('X2_Ehrenfest', 'X2_average'),
                  ('P_Ehrenfest', 'P_average'), ('P2_Ehrenfest', 'P2_average'),
                  ('XP_Ehrenfest', 'XP_average'), ('dPotentialdX_Ehrenfest', 'dPotentialdX_average'),
                  ('PdPotentialdX_average', 'PdPotentialdX_average'),
                  ('XdPotentialdX_average', 'XdPotentialdX_average'),
                  ('Hamiltonian_average', 'Hamiltonian_average'))


def wigner_tail(f, inst, extra=()):
    """What ``Run`` writes after the loop (GPU_Wigner2D_FFT.py:1936-1959;
    GPU_Wigner2D_GPitaevskii.py:2021-2048 adds ProbabilitySquare_average)."""
    f['timeRange'] = inst.timeRange
    f['timeRangeIndexSaved'] = np.asarray(inst.timeRangeIndexSaved)
    for key, attr in EHRENFEST_KEYS + tuple(extra):
        f['/Ehrenfest/' + key] = getattr(inst, attr)
    f['W_init'] = np.real(np.asarray(inst.W_init))
    f['W_end'] = inst.W_end
    f['negativeArea'] = inst.negativeArea


def load_ehrenfest(inst, fileName):
    """``LoadEhrenfestFromFile`` (GPU_Wigner2D_FFT.py:919-940)."""
    f = open_read(fileName)
    try:
        for key, attr in EHRENFEST_KEYS:
            setattr(inst, attr, np.array(f['/Ehrenfest/' + key][...]))
        inst.W_init = np.array(f['W_init'][...]) + 0j
        inst.W_end = np.array(f['W_end'][...]) + 0j
    finally:
        f.close()


# ---------------------------------------------------------------- Dirac layout
def dirac_header(f, inst):
    """The datasets ``GPU_Dirac2D.Run`` writes before the loop (GPU_Dirac2D.py:989-1006)."""
    f['x_gridDIM'], f['y_gridDIM'] = inst.X_gridDIM, inst.Y_gridDIM
    f['x_amplitude'], f['y_amplitude'] = inst.X_amplitude, inst.Y_amplitude
    f['dx'], f['dy'] = inst.dX, inst.dY
    for k in range(4):
        name = 'Potential_%d_String' % k
        f[name] = getattr(inst, name)


def dirac_density(psi):
    """``save_Density``: fftshift(sum_k |psi_k|^2) as float32."""
    rho = sum(np.abs(psi[k]) ** 2 for k in range(4))
    return np.ascontiguousarray(np.fft.fftshift(rho).astype(np.float32))


def dirac_frame(mode):
    def emit(f, key, psi):
        if mode == 'Spinor':                   # save_Spinor: '<component>/real|imag/<t>'
            for k in range(4):
                f['%d/real/%s' % (k + 1, key)] = psi[k].real
                f['%d/imag/%s' % (k + 1, key)] = psi[k].imag
            return psi
        rho = dirac_density(psi)
        f[str(key)] = rho
        return rho
    return emit


def dirac_frame_nosink(mode):
    """Frame formation without a file (``frames`` only)."""
    if mode == 'Spinor':
        return lambda f, key, psi: psi
    return lambda f, key, psi: dirac_density(psi)


# ---------------------------------------------------------------- Dirac3D layout
def dirac3_header(f, inst):
    """The datasets ``GPU_Dirac3D.Run`` writes before the loop (GPU_Dirac3D.py:1279-1293),
    with the z values under the z keys (the reference stores the y values there)."""
    f['x_gridDIM'], f['y_gridDIM'], f['z_gridDIM'] = inst.X_gridDIM, inst.Y_gridDIM, inst.Z_gridDIM
    f['x_amplitude'], f['y_amplitude'], f['z_amplitude'] = inst.X_amplitude, inst.Y_amplitude, inst.Z_amplitude
    f['dx'], f['dy'], f['dz'] = inst.dX, inst.dY, inst.dZ
    for k in range(4):
        name = 'Potential_%d_String' % k
        f[name] = getattr(inst, name)


def dirac3_frame(mode, to_file=True):
    """``save_Density`` (fftshift of sum_k |psi_k|^2 as float32) or, in ``'Spinor'`` mode,
    ``save_Spinor_SliceYZ`` at slice 0, 0: ``'xy/<k>/real|imag/<t>'`` = psi_k[0, :, :] and
    ``'xz/<k>/real|imag/<t>'`` = psi_k[:, 0, :] (GPU_Dirac3D.py:1041-1094).  The frame kept
    in memory is the density, or the pair of slice arrays."""
    def emit(f, key, psi):
        if mode == 'Spinor':
            xy, xz = np.array(psi[:, 0, :, :]), np.array(psi[:, :, 0, :])
            if to_file:
                for k in range(4):
                    for plane, arr in (('xy', xy), ('xz', xz)):
                        f['%s/%d/real/%s' % (plane, k + 1, key)] = arr[k].real
                        f['%s/%d/imag/%s' % (plane, k + 1, key)] = arr[k].imag
            return xy, xz
        rho = dirac_density(psi)
        if to_file:
            f[str(key)] = rho
        return rho
    return emit
