/* TEST INFRASTRUCTURE ONLY. Stand-in for <GL/gl.h> so the reference's
 * kernels/cudaPBF.cu (which includes cuda_gl_interop.h) compiles headless: the
 * GL type names come from the reference's vendored glad header; no GL function
 * is declared or linked. */
#ifndef PBF_ORACLE_GL_SHIM_H
#define PBF_ORACLE_GL_SHIM_H
#include <glad/glad.h>
#endif
