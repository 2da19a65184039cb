"""B200-native (sm_100a) collision operator and DP5(4) stepper for TORTOISE-style
Boltzmann transport on P1-DG simplex meshes.  See include/tortoise_b200.h."""
from .abi import BOSON, FERMION, IN, OUT  # noqa: F401
from .model import (Band, Material, MaterialStatus, MaterialTimeStatus, Mesh, Region,  # noqa: F401
                    ScatteringChannel)
