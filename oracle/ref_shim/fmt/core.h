// Empty stand-in: the reference's generate_csr.hpp includes <fmt/core.h> but
// calls nothing from it.  Used only by the oracle/_ref/ref_gen build.
#pragma once
