from cmmdft_b200.units import avogadro, boltzmann, planck, lightspeed  # noqa: F401
