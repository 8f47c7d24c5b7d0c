// Headless stand-in for the reference viewer's GLFW input manager: the camera class only
// queries these three getters while it is driven by keyboard or mouse, which a headless
// run never does.
#pragma once
#include <glm/glm.hpp>
class InputManager {
public:
    static glm::vec3 getMovementVector() { return glm::vec3(0.0f); }
    static glm::vec2 getMouseDelta() { return glm::vec2(0.0f); }
    static int getMouseScrollDelta() { return 0; }
};
