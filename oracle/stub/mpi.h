// Same single-process stand-in as petscsys.h (the reference headers include either name).
#pragma once
#include "petscsys.h"
