// Oracle build of the reference: MPI disabled (world size 1).
#pragma once
