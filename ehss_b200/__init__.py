"""ehss_b200: the SCIMMS/EHSS PA + EHSS cross-section path on B200 (sm_100a).

Public API (reference counterparts in parentheses):

* ``Spheres``, ``EHSSSource``, ``EHSSResult``  (inside_out_pa / ehss_state types)
* ``external_source``                            (ehss_state.external_source)
* ``PreparedStaticGPUEHSS(...).engine.trace``    (PreparedStaticCPUEHSS(...).engine.trace)
* ``SphereIndex(...).query``                     (pa_spatial.SphereIndex.query)
* ``CompactBoundary.fit(...).source``             (ehss_compact_source.CompactBoundary)
* ``Scene``, ``blocks.BlockPlan``                 fused Sobol -> trace -> reduction on the device
* ``ccs_cli``                                     the ccs.py calculation surface

Every computation runs in libehss_b200.so (hand-written CUDA for sm_100a);
importing this package needs no GPU, calling it does.
"""
from .state import EHSSResult, EHSSSource, Spheres
from .engine import (GPUEHSSTransport, PreparedStaticGPUEHSS, Scene, SphereIndex, external_source)
from .compact import CompactBoundary

__all__ = ['EHSSResult', 'EHSSSource', 'Spheres', 'GPUEHSSTransport', 'PreparedStaticGPUEHSS', 'Scene',
           'SphereIndex', 'external_source', 'CompactBoundary']
__version__ = '0.1.0'
