/* Empty stand-in for the MATLAB engine header included by the reference's
 * main.h (CODE/C++/VS2010/simLB/simLB/main.h:12); nothing from it is used. */
#ifndef REFSHIM_ENGINE_H_
#define REFSHIM_ENGINE_H_
#endif
