// Stand-in for the reference's device/printf.hpp (a debug printf into a Metal
// buffer): the host build of the reference's device code prints nothing.
#pragma once
#define printf(...) ((void)0)
