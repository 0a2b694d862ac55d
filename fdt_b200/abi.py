"""ctypes mirror of include/bpx.h (the structs and option defaults).

Kept free of any library loading so that tests can build option structs without a GPU.
"""
from __future__ import annotations

import ctypes as C

BPX_MAX_FIBRES = 3
BPX_NSTATE = 15

BPX_OK = 0
BPX_ERR_INVALID_ARG = 1
BPX_ERR_CUDA = 2
BPX_ERR_NO_DEVICE = 3
BPX_ERR_UNSUPPORTED = 4
BPX_ERR_IO = 5
BPX_ERR_BAD_DATA = 6

BPX_VOX_NONFINITE_DATA = 1
BPX_VOX_F0_REFIT = 2
BPX_VOX_NONFINITE_ENERGY = 4
BPX_VOX_LM_ITERATION_CAP = 8


def nrec(nfib: int) -> int:
    return 6 + 3 * nfib


class Options(C.Structure):
    """bpx_options: the xfibresOptions fields acting on the per-voxel path."""

    _fields_ = [
        ("model", C.c_int32),
        ("nfibres", C.c_int32),
        ("fudge", C.c_float),
        ("njumps", C.c_int32),
        ("nburn", C.c_int32),
        ("sampleevery", C.c_int32),
        ("updateproposalevery", C.c_int32),
        ("no_ard", C.c_int32),
        ("all_ard", C.c_int32),
        ("nonlin", C.c_int32),
        ("cnonlin", C.c_int32),
        ("rician", C.c_int32),
        ("f0", C.c_int32),
        ("ardf0", C.c_int32),
        ("R_prior_mean", C.c_float),
        ("R_prior_std", C.c_float),
        ("R_prior_fudge", C.c_float),
        ("gradnonlin", C.c_int32),
        ("seed", C.c_uint64),
        ("mcmc_tpv", C.c_int32),
        ("mcmc_mpl", C.c_int32),
        ("reserved", C.c_int32 * 6),
    ]

    @classmethod
    def make(cls, **kw) -> "Options":
        """xfibres defaults (xfibresoptions.h:104-149), overridden by ``kw``."""
        o = cls()
        o.model = 1
        o.nfibres = 1
        o.fudge = 1.0
        o.njumps = 1250
        o.nburn = 1000
        o.sampleevery = 25
        o.updateproposalevery = 40
        o.R_prior_mean = 0.13
        o.R_prior_std = 0.03
        o.R_prior_fudge = 0.0
        o.seed = 8665904
        for k, v in kw.items():
            if not hasattr(o, k):
                raise KeyError(k)
            setattr(o, k, v)
        return o

    @property
    def nparams_fit(self) -> int:
        return 2 + 3 * self.nfibres + (1 if self.model >= 2 else 0) + (1 if self.f0 else 0)

    @property
    def nsamples(self) -> int:
        return self.njumps // self.sampleevery


class Volume(C.Structure):
    _fields_ = [
        ("nvox", C.c_int32),
        ("ndir", C.c_int32),
        ("data", C.c_void_p),
        ("bvecs", C.c_void_p),
        ("bvals", C.c_void_p),
        ("grad", C.c_void_p),
        ("voxel_offset", C.c_uint64),
    ]


class Outputs(C.Structure):
    _fields_ = [
        ("th", C.c_void_p),
        ("ph", C.c_void_p),
        ("f", C.c_void_p),
        ("mean_d", C.c_void_p),
        ("mean_dstd", C.c_void_p),
        ("mean_R", C.c_void_p),
        ("mean_f0", C.c_void_p),
        ("mean_tau", C.c_void_p),
        ("mean_S0", C.c_void_p),
        ("mean_f", C.c_void_p),
        ("dyads", C.c_void_p),
        ("status", C.c_void_p),
    ]


class Item(C.Structure):
    """bpx_item: one volume of a batch."""

    _fields_ = [
        ("vol", Volume),
        ("model", C.c_int32),
        ("nfibres", C.c_int32),
        ("out", Outputs),
        ("mlp_params", C.c_void_p),
        ("nburn", C.c_int32),
        ("freeze_props", C.c_int32),
    ]


class PostProc(C.Structure):
    """bpx_postproc: the bedpostx_postproc arithmetic's outputs."""

    _fields_ = [
        ("mean_th", C.c_void_p),
        ("mean_ph", C.c_void_p),
        ("dispersion", C.c_void_p),
        ("dyads_thr", C.c_void_p),
        ("dyads_modf", C.c_void_p),
        ("mean_fsum", C.c_void_p),
    ]


class TrackOptions(C.Structure):
    """bpx_track_options: the probtrackx options of the simple mode (probtrackxOptions.h:198-236)."""

    _fields_ = [
        ("nparticles", C.c_int32),
        ("nsteps", C.c_int32),
        ("steplength", C.c_float),
        ("c_thr", C.c_float),
        ("fibthresh", C.c_float),
        ("distthresh", C.c_float),
        ("randfib", C.c_int32),
        ("fibst", C.c_int32),
        ("usef", C.c_int32),
        ("sampvox", C.c_int32),
        ("seed", C.c_uint64),
        ("pathdist", C.c_int32),
        ("loopcheck", C.c_int32),
        ("modeuler", C.c_int32),
        ("per_seed", C.c_int32),
        ("reserved", C.c_int32 * 1),
    ]

    @classmethod
    def make(cls, **kw) -> "TrackOptions":
        """probtrackx defaults (-P 5000 -S 2000 --steplength 0.5 -c 0.2 --fibthresh 0.01), overridden by kw."""
        o = cls()
        o.nparticles, o.nsteps, o.steplength, o.c_thr, o.fibthresh = 5000, 2000, 0.5, 0.2, 0.01
        o.distthresh, o.randfib, o.fibst, o.usef, o.sampvox, o.seed = 0.0, 0, 1, 0, 0, 8665904
        for k, v in kw.items():
            if not hasattr(o, k):
                raise KeyError(k)
            setattr(o, k, v)
        return o


class TrackVolume(C.Structure):
    """bpx_track_volume: samples [nfib][nsamples][nz][ny][nx], mask [nz][ny][nx], voxel size in mm."""

    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("dx", C.c_float),
        ("dy", C.c_float),
        ("dz", C.c_float),
        ("nfib", C.c_int32),
        ("nsamples", C.c_int32),
        ("th", C.c_void_p),
        ("ph", C.c_void_p),
        ("f", C.c_void_p),
        ("mask", C.c_void_p),
        ("avoid", C.c_void_p),
        ("stop", C.c_void_p),
        ("waypoints", C.c_void_p),
        ("nwaypoints", C.c_int32),
        ("ntargets", C.c_int32),
        ("targets", C.c_void_p),
        ("seeds_to_targets", C.c_void_p),
        ("m2_ncols", C.c_int32),
        ("lr_nx", C.c_int32),
        ("lr_ny", C.c_int32),
        ("lr_nz", C.c_int32),
        ("lr_dx", C.c_float),
        ("lr_dy", C.c_float),
        ("lr_dz", C.c_float),
        ("m2_lookup", C.c_void_p),
        ("matrix2", C.c_void_p),
        ("m1_ncols", C.c_int32),
        ("m1_lookup", C.c_void_p),
        ("matrix1", C.c_void_p),
        ("prefdir", C.c_void_p),
    ]
