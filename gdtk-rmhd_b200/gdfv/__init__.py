"""gdfv -- B200 (sm_100a) explicit structured-grid finite-volume update with the
solver options of Eilmer-4 / chicken (ausmdv, hllc, MHD hlle with GLM psi
cleaning; l2r2 van Albada reconstruction; predictor-corrector update).

All computation runs in libgdfv.so (CUDA); this package is the host side.
"""
from ._lib import GdfvError, exported_symbols, lib
from .solver import (Config, ExchangeBC_FullFace, FlowState, IdealGas, InFlowBC_Supersonic,
                     OutFlowBC_FixedP, OutFlowBC_FixedPT, OutFlowBC_SimpleExtrapolate, OutFlowBC_SimpleFlux,
                     Simulation, WallBC_WithSlip, FACE_INDEX, FACE_NAMES)

__all__ = ["Config", "ExchangeBC_FullFace", "FlowState", "IdealGas", "InFlowBC_Supersonic",
           "OutFlowBC_SimpleExtrapolate", "OutFlowBC_SimpleFlux", "OutFlowBC_FixedP", "OutFlowBC_FixedPT",
           "Simulation", "WallBC_WithSlip", "GdfvError",
           "exported_symbols", "lib", "FACE_INDEX", "FACE_NAMES"]
