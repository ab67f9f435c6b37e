"""B200-native exact BFS for implicit Cayley and permutation graphs.

Drop-in for the ``multigpubfs`` CayleyPy entry points (enable_native,
disable_native, bfs, NativeOptions, NativeBfsResult, run_graph,
GraphDefinition, from_cayleypy).  All search work runs in libmgbfs2 on the GPU;
importing the package has no side effects and loads no native code.
"""
from .graph_definition import GraphDefinition, from_cayleypy
from .launch import run_graph
from .cayleypy_backend import NativeOptions, NativeBfsResult, bfs, enable_native, disable_native

__all__ = ["GraphDefinition", "from_cayleypy", "run_graph", "NativeOptions", "NativeBfsResult", "bfs",
           "enable_native", "disable_native"]
