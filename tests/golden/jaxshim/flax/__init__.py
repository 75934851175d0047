"""Stand-in for the one piece of ``flax`` the reference's encrypted model
files use: ``nnx.Module`` as a plain base class (``nn_tfhe/Spike_LSTM.py``
subclasses it and keeps its arrays as attributes).  Used only to execute
those files for golden fixtures."""
from . import nnx  # noqa: F401
