def get_cmap(name=None, lut=None):
    return lambda *a, **k: (0.0, 0.0, 0.0, 1.0)
