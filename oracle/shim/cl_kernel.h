// Test infrastructure only.  Empty stand-in for the header that
// ConvexCell.cl:9 includes; the shim prelude already provides every OpenCL
// builtin the reference kernels use.
