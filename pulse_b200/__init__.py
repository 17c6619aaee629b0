"""B200 (sm_100a) CUDA implementation of pulse's path-tracing hot path.

The compute runs in ``libpulse_cuda.so`` (built from ``pulse_b200/csrc`` by
``pulse_b200.build``) behind the C ABI of ``include/pulse_cuda.h``; this
package holds its ctypes front end (``tracer``), the std430 scene layout
(``layout``), the host-side mirror of the reference's plugin interface
(``plugin``) and the seeded workload generators (``scenes``).
"""
__version__ = "0.1.0"
