/* Force-included when oracle/Makefile compiles the reference's own
 * kernels.cu and TGV2_kernels.cu for the B200 (target ref_gpu; test and
 * baseline infrastructure only).  The reference's exception.h overrides
 * std::exception::what() without noexcept, which current compilers reject; it
 * is not on the compute path, so its include guard is defined here and the
 * one macro its memory helpers use is supplied. */
#ifndef MVS_REF_GPU_PRELUDE_H
#define MVS_REF_GPU_PRELUDE_H
#include <iostream>
#include <stdexcept>
#include <string>
#define EXCEPTION_H
#define THROW_EXCEP(msg) throw std::runtime_error(std::string("reference: ") + (msg))
#endif
