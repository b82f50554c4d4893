// Oracle build of the reference: no MKL, MPI, cereal, ranges-v3 or METIS.
#pragma once
