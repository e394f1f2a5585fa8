/* Compile-only stand-in for <GL/glew.h>, used only when building the
 * reference's code into oracle/_ref.  The reference calls
 * glEnable/glBlendFunc/glWindowPos2i only inside TypicalRayProducer::RenderImage,
 * which draws nothing the projector computes, and ST_Tomography.cpp loads its
 * view and projection matrices into the GL matrix stack and clears the frame
 * buffer (ST_Tomography.cpp:654-658, 814-816, 926-929): none of that feeds a
 * computed value (the projector reads the matrices from the scene object).
 * These no-ops keep those files compilable without any graphics library; no
 * GL library is linked or loaded. */
#ifndef STT_ORACLE_SHIM_GLEW_H
#define STT_ORACLE_SHIM_GLEW_H
#define GL_BLEND 0x0BE2
#define GL_ONE 1
#define GL_ONE_MINUS_SRC_ALPHA 0x0303
#define GL_MODELVIEW 0x1700
#define GL_PROJECTION 0x1701
#define GL_DEPTH_BUFFER_BIT 0x00000100
#define GL_COLOR_BUFFER_BIT 0x00004000
static inline void glEnable(unsigned) {}
static inline void glBlendFunc(unsigned, unsigned) {}
static inline void glWindowPos2i(int, int) {}
static inline void glViewport(int, int, int, int) {}
static inline void glMatrixMode(unsigned) {}
static inline void glLoadMatrixf(const float *) {}
static inline void glClearColor(float, float, float, float) {}
static inline void glClearDepth(double) {}
static inline void glClear(unsigned) {}
static inline unsigned glewInit(void) { return 0; }
#endif
