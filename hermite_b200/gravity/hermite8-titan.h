// hermite8-titan.h -- drop-in for the reference's SRC/hermite8-titan.h:
// SRC/hermite8.h includes this file under -DCUDA_TITAN; the Gravity it
// declares runs on the hermite_b200 library.
#pragma once
#define HB_GRAVITY_ORDER 8
#include "hb_gravity.inl"
