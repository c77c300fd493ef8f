/* Type stubs so that the reference's CUDA engine compiles without a
 * graphics stack: its GL-interop entry points are never called here. */
#pragma once
typedef unsigned int GLuint;
typedef unsigned int GLenum;
#define GL_TEXTURE_2D 0x0DE1
