// LAMMPS header name mapped onto the shim
#pragma once
#include "lammps_shim.h"
