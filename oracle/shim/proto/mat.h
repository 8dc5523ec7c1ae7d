// Test infrastructure (oracle): 3x3 matrices live with the vectors (proto/vec.h).
#pragma once

#include "proto/vec.h"
