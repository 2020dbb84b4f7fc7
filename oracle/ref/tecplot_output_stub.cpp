// Replaces the reference's tecplot_output.cpp in the oracle build.
//
// That file only writes Tecplot .plt files through the closed TECIO library,
// which is absent here. For <type>spring_network</type> objects its
// tecplot_output_lagrangian_object (called once by program.cpp:76) also sizes
// arrays from object.radial_nodes / depth_nodes (tecplot_output.cpp:533-535,
// 667-691), which only the rigid_cylinder path initialises
// (lagrangian_object.cpp:79-113); with them uninitialised the allocation
// fails. Every method here is therefore a no-op: no solver arithmetic or state
// flows through Tecplot output.
#include "tecplot_output.h"

template <typename T> tecplot_output<T>::tecplot_output() {}
template <typename T>
tecplot_output<T>::tecplot_output(global_variables&, Mesh&, Solution&, Boundary_Conditions&, int,
                                  double, post_processing&) {}
template <typename T> tecplot_output<T>::~tecplot_output() {}
template <typename T>
void tecplot_output<T>::tecplot_output_unstructured_soln(global_variables&, unstructured_mesh&,
                                                         Solution&, Boundary_Conditions&, double,
                                                         post_processing&, Solution&, double*,
                                                         T*) {}
template <typename T>
void tecplot_output<T>::tecplot_output_lagrangian_object(lagrangian_object&, global_variables&,
                                                         domain_geometry&, double) {}
template <typename T>
void tecplot_output<T>::tecplot_output_lagrangian_object_gpu(double*, double*, double*, double*,
                                                             double*, double*, double*, double*,
                                                             double*, global_variables&,
                                                             domain_geometry&, double,
                                                             std::string, int, int, int) {}
// tecplot_output.h itself ends with the explicit instantiations for float and double.
