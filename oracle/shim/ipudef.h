/* Empty stand-in for the Poplar SDK's <ipudef.h> (TEST INFRASTRUCTURE). */
#pragma once
