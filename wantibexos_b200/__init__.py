"""B200-native (sm_100a) Bethe-Salpeter exciton + optics path of WanTiBEXOS.

The compute path is libwtbgpu.so (hand-written CUDA, C-ABI in include/wtbgpu.h);
``wtbgpu`` binds it from Python and ``synth`` generates the seeded synthetic models.
"""
__all__ = ["wtbgpu", "synth"]
