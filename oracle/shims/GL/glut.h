/* Compile-only stand-in for <GL/glut.h> (oracle/_ref build only): Scene::Resize
 * calls glViewport, which has no effect on any computed value. */
#include "glew.h"
