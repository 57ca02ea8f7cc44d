// Stand-in for the reference's device/printf.hpp (a debug printf into a Metal
// buffer): none of the compiled device code prints, so the host build needs
// nothing from it.
#pragma once
