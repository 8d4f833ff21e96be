"""B200-native Kim-Moin-Moser channel timestep (drop-in for ryankellybp11/Polymer_DNS's hot path)."""
from . import abi  # noqa: F401
