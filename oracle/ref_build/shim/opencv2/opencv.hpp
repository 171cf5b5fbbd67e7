// The reference includes OpenCV but every use on the compiled files is
// commented out; only the namespace it imports must exist.
#pragma once
namespace cv {}
