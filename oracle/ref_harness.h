// Test infrastructure (oracle): the scene handle shared by the two checker
// libraries.  libsol_ref.so (ref_harness.cpp) builds and renders sol::Scene
// objects with SoL's own code only; libsol_dropin.so (dropin_harness.cpp)
// renders the same handles through the GPU drop-in and links the product
// library, so that timing SoL's CPU path never maps the product.
#pragma once

#include "sol/scene.h"

struct RefScene {
    sol::Scene scene;
};

extern "C" {
/// Sets the text ref_last_error() returns on this thread.
void ref_set_error(const char* what);
}
