"""B200 (sm_100a) CUDA implementation of pulse's path-tracing hot path.

The compute runs in ``libpulse_cuda.so`` (built from ``pulse_b200/csrc`` by
``pulse_b200.build``) behind the C ABI of ``include/pulse_cuda.h``; this
package holds its ctypes front end (``tracer``), the std430 scene layout
(``layout``), the seeded workload generators (``scenes``), the launch-shape
autotuner (``autotune``) and the differentiable-rendering helpers (``diff``).
The host-side mirror of the reference's plugin interface is C++
(``host/pulse_plugin.hpp``, built as ``libpulse_plugin.so``).
"""
__version__ = "0.1.0"
