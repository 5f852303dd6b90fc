"""Small helpers shared with the reference's on-disk conventions."""
from .units import kjmol

__all__ = ['get_file_suffix', 'convert_units', 'Document']


def get_file_suffix(chempot, temp):
    """File suffix of density files, e.g. ``-36.84600kJmol_300.00000K``
    (cmmdft/tools.py:64-79)."""
    if hasattr(chempot, '__iter__'):
        s = ''
        for mu in chempot:
            s += f'{mu / kjmol:#7.5f}kJmol_'
        return s + f'{temp:#7.5f}K'
    return f'{chempot / kjmol:#7.5f}kJmol_{temp:#7.5f}K'


class convert_units(object):
    """Loading-unit conversions for one guest and host (cmmdft/tools.py:368-399):
    mass_guest in atomic units, mass_host the host cell's mass in atomic
    units, volume_host in bohr^3.  ``conversion_factor(input, output)``
    multiplies a loading in ``input`` units into ``output`` units; the units
    are 'wt%', 'mg/g', 'cm3/cm3', 'mol/mol', 'mol/g', 'mol/kg' and 'au/uc'
    (molecules per unit cell)."""
    UNITS = ('wt%', 'cm3/cm3', 'mol/mol', 'mol/g', 'mol/kg', 'au/uc', 'mg/g')

    def __init__(self, mass_guest, mass_host, volume_host):
        from .units import amu, gram, centimeter
        rho_stp = (mass_guest / amu) * 1e-3 / 22.414            # g/cm^3 of the gas at STP
        rho_host = (mass_host / gram) / (volume_host / centimeter ** 3)
        self.per_unit = {'wt%': mass_host / mass_guest / 100, 'mg/g': mass_host / mass_guest / 1000,
                         'cm3/cm3': mass_guest * rho_host / mass_host / rho_stp, 'mol/mol': 1,
                         'mol/g': mass_host / amu, 'mol/kg': mass_host / amu / 1000, 'au/uc': 1}

    def conversion_factor(self, input='mol/mol', output='mol/mol'):
        assert input in self.UNITS and output in self.UNITS, "unknown loading unit"
        return self.per_unit[input] / self.per_unit[output]


class Document(object):
    """A minimal writer of the Adsorption Information File format (CIF-like
    text): named data blocks of key/value pairs followed by loops of columns,
    written as the reference's AIF export does (cmmdft/tools.py:401-458)."""

    class Block(object):
        def __init__(self, name):
            self.name = name
            self.pairs = {}
            self.loops = []

        def set_pair(self, key, value):
            self.pairs[key] = value

        def init_loop(self, prefix, keys):
            loop = Document.Loop(prefix, keys)
            self.loops.append(loop)
            return loop

    class Loop(object):
        def __init__(self, prefix, keys):
            self.prefix, self.keys = prefix, list(keys)
            self.columns = {k: [] for k in self.keys}

        def set_all_values(self, columns):
            for k, col in zip(self.keys, columns):
                self.columns[k] = list(col)

    def __init__(self):
        self.blocks = []

    def add_new_block(self, name):
        self.blocks.append(Document.Block(name))
        return self.blocks[-1]

    def sole_block(self):
        return self.blocks[0] if self.blocks else self.add_new_block('default')

    def text(self):
        out = []
        for blk in self.blocks:
            out.append('data_%s' % blk.name)
            out.extend('%s %s' % (k, v) for k, v in blk.pairs.items())
            for loop in blk.loops:
                out.append('')
                out.append('loop_')
                out.extend(loop.prefix + k for k in loop.keys)
                n = len(loop.columns[loop.keys[0]]) if loop.keys else 0
                out.extend(''.join(loop.columns[k][i] + ' ' for k in loop.keys) for i in range(n))
        return '\n'.join(out) + '\n'

    def write_file(self, path):
        with open(path, 'w') as f:
            f.write(self.text())
