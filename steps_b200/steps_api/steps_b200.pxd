# Cython declaration of the drop-in solver steps::b200::TetOpSplitB200
# (steps_api/tetopsplit_b200.hpp) for STEPS' own Cython build (pysteps/): the binding
# module cysteps_b200.pyx cimports it, as cysteps_mpi.pyx cimports TetOpSplitP from
# steps_mpi.pxd (pysteps/steps_mpi.pxd:63-65).
from libcpp.memory cimport shared_ptr
cimport std
cimport steps
cimport steps_model
cimport steps_wm
cimport steps_rng

cdef extern from "steps_api/tetopsplit_b200.hpp" namespace "steps::b200":
    cdef cppclass TetOpSplitB200:
        TetOpSplitB200(steps_model.Model*, steps_wm.Geom*, shared_ptr[steps_rng.RNG], int,
                       std.vector[int], std.map[steps.triangle_global_id, int], std.vector[int]) except +
        std.string getSolverName() except +
        std.string getSolverDesc() except +
        std.string getSolverAuthors() except +
        std.string getSolverEmail() except +
        void checkpoint(std.string) except +
        void restore(std.string) except +
        void reset() except +
        void run(double) except +
        void advance(double) except +
        void step() except +
        double getTime() except +
        unsigned int getNSteps() except +
        void setTemp(double) except +
        double getTemp() except +
        void setEfieldDT(double) except +
        double getEfieldDT() except +
        void getBatchTetSpecCountsNP(steps.index_t*, size_t, std.string, double*, size_t) except +
