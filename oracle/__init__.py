"""CPU oracle of the stencil path -- test infrastructure only.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg;
never by the cutile package.  See stencil_oracle.py.
"""
