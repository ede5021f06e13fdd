"""mcstar_b200 -- B200-native conserved phase-field-crystal stepper.

Host-side mirror of the mcstar-libs header API over the C ABI of libpfc_b200.so
(include/pfc_b200.h).  The CUDA kernels (sm_100a) do all device work; torch is used
for device memory and streams only.
"""
from ._lib import PfcError, LIB_PATH, lib
from .array import GPUArray, CPUArray, AsReal, AsCmpl, shape_tr
from .context import Context, get_context, tune
from .kernels import (CufftPlan, R2C, C2R, NoiseHostApi, call_kernel_update_eom, call_kernel_update_eom_with_fen,
                      call_kernel_calc_fen, call_kernel_psi3_split, call_kernel_norm, call_kernel_findpeaks,
                      call_kernel_findpeaks_2d, bond_order_analysis, write_bond_table, maximum_dtype, Maximum,
                      mu, omega, init_pot_line, TimeAcc, BOND_COLUMNS, findpeaks_device, records_to_host)
from .stepper import Stepper, liquid_random, bcc_sphere, namp_from_temperature, BCC_Q
from .ensemble import Ensemble, ensemble_members, partition, member_cost
from .adjoint import AdjointRun, SFLoss, structure_factor
from . import dist

__all__ = [n for n in dir() if not n.startswith("_")]
