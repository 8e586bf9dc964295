// Forwards to the OpenMP-backed TBB stand-in (test infrastructure only).
#pragma once
#include "tbb.h"
