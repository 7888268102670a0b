/* empty stand-in (test infrastructure only) */
#pragma once
