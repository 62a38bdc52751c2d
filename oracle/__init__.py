"""CPU oracle of the uniform-grid PF-FLIP step — test infrastructure only.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline legs,
always as the checker or the timed CPU baseline; the product (the pfflip
package and libpfflip.so) never imports it.
"""
