// placeholder until the HEM sources land
