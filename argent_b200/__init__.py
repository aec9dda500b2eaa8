"""argent_b200 — a B200-native (sm_100a) replacement for argent's spectral
path-tracing hot path (`render_pass` / `trace`, crates/argent-core/src/render.rs
and integrator.rs), behind a C ABI (include/argent_gpu.h)."""

from . import _native  # noqa: F401
