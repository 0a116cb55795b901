"""B200 (sm_100a) physical-optics diffraction for MBS-fast.

Drop-in for the reference's HandlerPO GPU entry points: beams from the
reference's host tracer go through the C ABI in include/mbs_po_b200.h to
hand-written CUDA kernels.
"""
