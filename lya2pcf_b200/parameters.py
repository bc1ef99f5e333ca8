"""Module-level constants of the lya2pcf configuration, under the names the
reference's drivers star-import (``from parameters import *``).

Values follow lya2pcf ``parameters.py:7-65``. The names must stay identical
because the drivers (``2pla.py``, ``distortion.py``) and ``post_processing.py``
read them unqualified; the values are the reference defaults.  Two entries are
informational only in this implementation:

* ``max_lenght`` -- the reference pads every forest to this many pixels and
  ``delta_reader.py:148`` rewrites it in place.  This implementation stores
  forests unpadded (CSR), so the value is not needed and is kept only so code
  that prints or forwards it keeps working.
* ``number_of_neighs`` -- the reference sizes its distortion scratch for this
  many neighbours (``distortion_procedures_pycuda.py:170-185``) and silently
  overruns it when more are kept.  Here scratch is sized from the data.
"""
import numpy as np

# I/O locations (parameters.py:10-11)
data_dir = './deltas_lya2pcf/'
corr_dir = './outputs/test/'
delta_key = "DELTA"

# Histogram geometry (parameters.py:18-25)
bin_size_r = 4          # Mpc/h
rmax = 200              # Mpc/h
rpmax = rmax
rtmax = rmax
numpix_rp = rpmax // bin_size_r
numpix_rt = rtmax // bin_size_r
numpix_mu = 10
numpix_theta = 10
numpix_r = rmax // bin_size_r

# Physical constants (parameters.py:30-34)
lambdaa = 1215.67       # Lyman-alpha rest wavelength, Angstrom
la = np.log10(lambdaa)
c = 299792.458          # km/s
halfpi = np.pi / 2

# Forest parameters (parameters.py:37-42)
gamma = 3.8
gammaovertwo = gamma / 2
z_ref = 2.25
nside = 32
chiquito = 2. / 3600. * 3.14159 / 180.   # 2 arcsec small-angle switch of the CPU kernel

# Cosmology (parameters.py:44-51)
Omm = 0.3153
OmDE = 1. - Omm
d_H0 = c / 100          # Mpc/h
zmin = 0
zmax = 10
nz = 10000

# Launch shapes of the reference PyCUDA kernels (parameters.py:55-59); kept for
# callers that forward them, unused by this implementation.
threads_per_block = (8, 32, 4)
threads_per_block_2 = (32, 32, 1)
max_threads = 1024

max_lenght = np.int32(208)
number_of_neighs = 80

# Multi-device placement (parameters.py:64-65)
number_of_cuda_devices = 4
cuda_device_first_number = 0
