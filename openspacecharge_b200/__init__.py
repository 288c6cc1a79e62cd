"""B200-native space-charge step of OpenSpaceCharge: CIC deposition, IGF free-space /
cathode-image / rectangular-pipe Green functions, doubled-grid FFT convolution, E on the
grid and interpolation back to particles, as hand-written sm_100a CUDA kernels behind a
C ABI (``include/opensc_gpu.h``, ``libopensc_b200.so``).
"""
from .native import (DEPOSIT_ATOMIC, DEPOSIT_DETERMINISTIC, DEPOSIT_SORTED_SEGMENT, OPT_BATCH_GRAPH, OPT_CHECK_FINITE,
                     OPT_DEPOSIT_MODE, OPT_GREEN_CACHE_MB, OPT_PARTICLE_ORDER, OPT_PRECISION, OPT_PROFILE, OPT_VJP_REUSE_FORWARD,
                     OPT_STRICT_BOUNDS, ORDER_ANY, ORDER_CELL_SORTED, ORDER_SORT,
                     PREC_FP32, PREC_FP64, PREC_FP64_PLAIN, Context, OscBunch, OscError, OscMesh3D)
from .mesh import (Mesh3D, batch_space_charge_step, batch_space_charge_step_dev, depose_rho_scalar, deposit_particles, get_mesh_quantities,
                   interpolate_field, osc_freespace_solver2, osc_read_rectpipe_grn,
                   osc_rectpipe_green, osc_write_rectpipe_grn, space_charge_3d,
                   space_charge_cathodeimages, space_charge_freespace, space_charge_rectpipe,
                   space_charge_step, space_charge_step_dev, space_charge_step_rectpipe_dev, write_lines, write_plane,
                   format_1pe14_7, sort_particles_dev, cell_keys)
from . import bunch

__version__ = "0.1.0"
