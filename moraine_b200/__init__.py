"""moraine_b200 — the distributed-scatterer chain of Moraine on NVIDIA B200 (sm_100a).

Drop-in replacements for ``moraine.shp``, ``moraine.co``, ``moraine.pl``, ``moraine.pqm``,
``ras2pc`` / ``pc2ras`` of ``moraine.pc`` and the pair ordering of ``moraine.tnet``: same
names, arguments and array layouts, run by hand-written CUDA kernels behind the C ABI in
``include/moraine_b200.h``.
"""
from .calamp import calamp, rslc2amp
from .co import ad_intf_pc, emperical_co, emperical_co_pc, uncompress_coh
from .pc import ds_candidates, pc2ras, ras2pc
from .pl import ds_temp_coh, emi, emperical_co_emi_temp_coh_pc
from .pqm import temp_coh
from .ps import amp_disp
from .shp import ks_test, select_shp
from .tnet import TempNet, nimage_from_npair

__version__ = "0.1.0"

__all__ = [
    "ks_test", "select_shp", "emperical_co", "emperical_co_pc", "ad_intf_pc", "uncompress_coh", "emi", "ds_temp_coh",
    "emperical_co_emi_temp_coh_pc", "temp_coh", "TempNet", "nimage_from_npair", "amp_disp", "rslc2amp", "calamp",
    "ras2pc", "pc2ras", "ds_candidates",
]
