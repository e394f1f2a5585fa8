/* Compile-only stand-in for <GL/glew.h>, used only when building the
 * reference's projector core into oracle/_ref.  The reference calls
 * glEnable/glBlendFunc/glWindowPos2i only inside TypicalRayProducer::RenderImage,
 * which draws nothing the projector computes.  These no-ops keep that file
 * compilable without any graphics library; no GL library is linked or loaded. */
#ifndef STT_ORACLE_SHIM_GLEW_H
#define STT_ORACLE_SHIM_GLEW_H
#define GL_BLEND 0x0BE2
#define GL_ONE 1
#define GL_ONE_MINUS_SRC_ALPHA 0x0303
static inline void glEnable(unsigned) {}
static inline void glBlendFunc(unsigned, unsigned) {}
static inline void glWindowPos2i(int, int) {}
static inline void glViewport(int, int, int, int) {}
static inline unsigned glewInit(void) { return 0; }
#endif
