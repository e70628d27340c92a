// Empty stand-in (test infrastructure): the reference header that includes
// this uses nothing from it in the code compiled by oracle/build_ref.sh.
#pragma once
