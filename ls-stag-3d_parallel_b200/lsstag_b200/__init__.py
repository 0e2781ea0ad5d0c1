"""Host-side Python mirror of the LS-STAG-3D pressure-projection solver
interface, backed by the B200 C-ABI library ``liblsstag_b200.so``."""
