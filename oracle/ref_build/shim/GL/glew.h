// Type names only, so that the reference's headers (which name GLuint in
// structs) compile as host C++.  No GL function is declared or provided.
#pragma once
typedef unsigned int GLuint;
typedef int GLint;
typedef unsigned int GLenum;
typedef char GLchar;
typedef int GLsizei;
typedef float GLfloat;
