from .passes import LazyQubitReordering, Tile
from .pm import PassManager, make_custom_pm, tile_circuit

__all__ = ["LazyQubitReordering", "Tile", "PassManager", "make_custom_pm", "tile_circuit"]
