// psg_ns3d_f64.cu -- FP64 instantiation of the 3D engine (kernels for every grid size).
#include "psg_ns3d_impl.cuh"
psg::Engine3DBase* psg::make_engine3d_f64() { return new psg::Engine3D<double>(); }
