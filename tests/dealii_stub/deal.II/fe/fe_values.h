// Stand-in: see dealii_stub.h.
#pragma once
#include "../../dealii_stub.h"
