"""B200-native FESOM2 tracer advection step (do_oce_adv_tra) behind the
reference's tracer_c_interface C ABI.  See include/fesom_tracer.h."""
from .tracer import FESOMTracerAdvection, synth_bathymetry, synth_bathymetry_smooth  # noqa: F401
from ._lib import LIB_PATH, REFERENCE_SYMBOLS, load  # noqa: F401
