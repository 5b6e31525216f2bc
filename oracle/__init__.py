"""CPU oracle of the Siddon projector — test infrastructure only (tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline legs).  The product
package ct_laboratory_b200 never imports it."""
