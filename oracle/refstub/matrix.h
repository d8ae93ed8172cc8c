/* Empty stand-in for MATLAB's matrix.h (see mex.h in this folder). */
