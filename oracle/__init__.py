"""Test infrastructure: the oracle for SRF's listmode projector path.

Nothing in the shipped package imports this package. Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it, as the
checker. See ``oracle/srf_oracle.cpp`` for the C++ restatement of the projectors and
``oracle/preprocess_ref.py`` for the numpy restatement of the LOR preprocessing.
"""
