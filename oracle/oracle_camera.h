// Test infrastructure (oracle): sol::PerspectiveCamera constructor arguments
// (include/sol/cameras.h:37-42), as the checkers receive them.
#pragma once

struct OracleCamera {
    float eye[3], dir[3], up[3];
    float fov;      // horizontal field of view, degrees
    float aspect;   // width / height
};
