"""Small helpers shared with the reference's on-disk conventions."""
from .units import kjmol

__all__ = ['get_file_suffix']


def get_file_suffix(chempot, temp):
    """File suffix of density files, e.g. ``-36.84600kJmol_300.00000K``
    (cmmdft/tools.py:64-79)."""
    if hasattr(chempot, '__iter__'):
        s = ''
        for mu in chempot:
            s += f'{mu / kjmol:#7.5f}kJmol_'
        return s + f'{temp:#7.5f}K'
    return f'{chempot / kjmol:#7.5f}kJmol_{temp:#7.5f}K'
