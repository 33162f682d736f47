"""The reference's element table (the "affinity table").

Values follow ``ELEMENTS`` in src/physics/forces.rs:43-54 (sigma, epsilon in
kelvin, charge) and ``AtomType::mass`` in src/components/atom_type.rs:80-93.
The index order is ``element_index`` (src/physics/forces.rs:176-189).
"""
from __future__ import annotations

SYMBOLS = ("H", "He", "C", "N", "O", "Na", "Si", "P", "S", "Fe")
NAMES = ("Hydrogen", "Helium", "Carbon", "Nitrogen", "Oxygen", "Sodium",
         "Silicon", "Phosphorus", "Sulfur", "Iron")
ATOMIC_NUMBER = (1, 2, 6, 7, 8, 11, 14, 15, 16, 26)  # AtomType discriminants
SIGMA = (1.6, 1.4, 1.9, 1.7, 1.65, 2.0, 2.3, 2.2, 2.1, 1.9)
EPSILON_K = (12.0, 8.0, 80.0, 40.0, 55.0, 110.0, 200.0, 150.0, 130.0, 350.0)
CHARGE = (0.0, 0.0, 0.0, 0.0, -1.0, 1.0, 0.5, 0.0, 0.0, 1.0)
MASS = (1.008, 4.0026, 12.011, 14.007, 15.999, 22.99, 28.085, 30.974, 32.06, 55.845)
COUNT = 10

LJ_CUTOFF_FACTOR = 2.5   # src/physics/forces.rs:169
LJ_NUCLEUS = 0.5         # src/physics/forces.rs:173
BOND_FACTOR = 1.5        # src/analysis/mod.rs:20
G_SAMPLE_CAP = 8192      # src/analysis/mod.rs:28
DEBOUNCE = 2             # src/systems/bonds.rs:27


def by_name(name: str) -> int | None:
    """Element index for a symbol or full name (AtomType::by_name,
    src/components/atom_type.rs:35-49): exact symbol, capitalised or
    lower-case full name."""
    n = name.strip()
    for i, (s, full) in enumerate(zip(SYMBOLS, NAMES)):
        if n == s or n == full or n == full.lower():
            return i
    return None
