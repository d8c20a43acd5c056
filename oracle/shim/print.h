/* Empty stand-in for the Poplar SDK's <print.h> (TEST INFRASTRUCTURE). */
#pragma once
