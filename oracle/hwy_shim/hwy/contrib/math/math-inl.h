// Stand-in: the ops the reference needs from this header live in hwy/highway.h.
#pragma once
#include "hwy/highway.h"
