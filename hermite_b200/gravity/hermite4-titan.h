// hermite4-titan.h -- drop-in for the reference's SRC/hermite4-titan.h:
// SRC/hermite4.h includes this file under -DCUDA_TITAN; the Gravity it
// declares runs on the hermite_b200 library.
#pragma once
#define HB_GRAVITY_ORDER 4
#include "hb_gravity.inl"
