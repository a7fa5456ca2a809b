"""CPU oracle for the pFq CMF walk -- TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package, and only as the checker. The product library
(``cmfw``) never imports it.

Two checkers live here:

* ``liboracle.so`` -- this project's plain-C restatement of the reference
  walk (cmfw_oracle.c), bitwise identical to the reference's kernel bodies
  compiled for the host when both run unfused;
* ``_ref/libref_*.so`` -- the reference's own kernel bodies compiled for the
  host by ``make -C oracle ref`` (present only where the reference sources
  were available at build time; the built files travel with the tree).

``exact`` holds the exact rational walk (Python ``Fraction``) for small
cases; ``exact_check`` turns the C exact walk modulo primes
(``exact_residues``) into exact limit values (CRT and rational
reconstruction) and checks floating-point limits against them.
"""
from .ffi import (  # noqa: F401
    IN_DTYPE, OUT_DTYPE, OUT_F64_DTYPE, ORACLE_LIB, build, column, f64_snapshots,
    have_ref, make_inputs, mt64_stream, ref_f64_snapshots, ref_make_inputs,
    ref_rns_moduli, ref_rns_trace, ref_walk, rns_moduli, rns_trace, walk, walk_f64_src, exact_residues,
    have_ref_gpu, ref_gpu_launch,
)
