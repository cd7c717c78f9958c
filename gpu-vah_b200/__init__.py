"""B200 VAH time step: libvah.so (CUDA, sm_100a) and its Python binding.

The directory name is not a Python identifier; load it with
importlib (see __graft_entry__.py) or put this directory on sys.path and
``import vah``.
"""
from .vah import *  # noqa: F401,F403
