"""TEST INFRASTRUCTURE ONLY: CPU oracle for toaster's GPU path-tracing path.

A C++17 restatement (oracle.cpp) of the reference's CPU renderer and BVH
(crates/toaster-cpu, crates/toaster-bvh, crates/toaster-scene/src/environment.rs). Only the
tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference arm use it, and only
as the checker or the timed CPU baseline; the CUDA library never calls it.

The reference itself (Rust) cannot be built here: cargo/rustc are absent. Its known-answer
tests are restated in tests/test_oracle_known_answers.py to pin this restatement; image
parity against the reference is statistical because the reference's random stream
(rand 0.9.4 ChaCha12) is not reproduced.
"""

from .binding import Oracle, OracleEnvironment, build, library_path  # noqa: F401
