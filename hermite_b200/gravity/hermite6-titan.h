// hermite6-titan.h -- drop-in for the reference's SRC/hermite6-titan.h:
// SRC/hermite6.h includes this file under -DCUDA_TITAN; the Gravity it
// declares runs on the hermite_b200 library.
#pragma once
#define HB_GRAVITY_ORDER 6
#include "hb_gravity.inl"
